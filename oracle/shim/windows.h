/*
 * Test-harness shim, NOT product code: the handful of Win32 names that the
 * reference's platform layer (src/platform_win.h:23-160) uses, mapped onto
 * POSIX so the unmodified reference builds on Linux as the parity oracle and
 * the CPU baseline.  The reference includes <windows.h> and <malloc.h> with
 * angle brackets (src/platform_win.h:23-24), so `-I oracle/shim` picks these
 * files up without touching the reference's sources.
 *
 * Mapping (one line each):
 *   VirtualAlloc(MEM_RESERVE)  -> mmap(PROT_READ|PROT_WRITE, MAP_NORESERVE)
 *   VirtualAlloc(MEM_COMMIT)   -> no-op (pages are faulted in on first touch)
 *   VirtualAlloc(MEM_RESET)    -> madvise(MADV_DONTNEED) on the whole pages
 *   GetProcAddress             -> NULL (the reference then takes MEM_RESET)
 *   SRWLOCK / CONDITION_VARIABLE -> pthread_mutex_t / pthread_cond_t
 *   INIT_ONCE                  -> a mutex plus a done flag
 *   CreateThread               -> detached pthread_create
 *   Interlocked*               -> __atomic builtins (sequentially consistent)
 *   GetSystemInfo              -> sysconf(_SC_NPROCESSORS_ONLN), or the
 *                                 FF_CPUS environment variable when set
 *   QueryPerformance*          -> clock_gettime(CLOCK_MONOTONIC), ns ticks
 */
#ifndef FASTFIB_ORACLE_WINDOWS_SHIM_H
#define FASTFIB_ORACLE_WINDOWS_SHIM_H

#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <sys/mman.h>
#include <time.h>
#include <unistd.h>

typedef int BOOL;
typedef uint32_t DWORD;
typedef long LONG;
typedef void *PVOID;
typedef void *LPVOID;
typedef const char *LPCSTR;
typedef size_t SIZE_T;
typedef void *HANDLE;
typedef void *HMODULE;
typedef void (*FARPROC)(void);

#define WINAPI
#define CALLBACK
#define TRUE 1
#define FALSE 0
#define INFINITE 0xFFFFFFFFu

#define MEM_COMMIT 0x1000u
#define MEM_RESERVE 0x2000u
#define MEM_RESET 0x80000u
#define PAGE_READWRITE 0x04u

static inline void *VirtualAlloc(void *addr, SIZE_T bytes, DWORD type, DWORD prot) {
    (void)prot;
    if (type & MEM_RESERVE) {
        void *p = mmap(addr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        return p == MAP_FAILED ? NULL : p;
    }
    if (type & MEM_RESET) {
        uintptr_t lo = ((uintptr_t)addr + 4095) & ~(uintptr_t)4095;
        uintptr_t hi = ((uintptr_t)addr + bytes) & ~(uintptr_t)4095;
        if (hi > lo) madvise((void *)lo, hi - lo, MADV_DONTNEED);
        return addr;
    }
    return addr; /* MEM_COMMIT: the reservation is already readable and writable */
}

static inline HMODULE GetModuleHandleA(LPCSTR name) { (void)name; return NULL; }
static inline FARPROC GetProcAddress(HMODULE m, LPCSTR name) { (void)m; (void)name; return NULL; }

typedef pthread_mutex_t SRWLOCK;
#define SRWLOCK_INIT PTHREAD_MUTEX_INITIALIZER
static inline void AcquireSRWLockExclusive(SRWLOCK *l) { pthread_mutex_lock(l); }
static inline void ReleaseSRWLockExclusive(SRWLOCK *l) { pthread_mutex_unlock(l); }

typedef pthread_cond_t CONDITION_VARIABLE;
#define CONDITION_VARIABLE_INIT PTHREAD_COND_INITIALIZER
static inline BOOL SleepConditionVariableSRW(CONDITION_VARIABLE *c, SRWLOCK *l, DWORD ms, unsigned long flags) {
    (void)ms; (void)flags; /* the reference only waits with INFINITE */
    return pthread_cond_wait(c, l) == 0;
}
static inline void WakeConditionVariable(CONDITION_VARIABLE *c) { pthread_cond_signal(c); }
static inline void WakeAllConditionVariable(CONDITION_VARIABLE *c) { pthread_cond_broadcast(c); }

typedef struct {
    pthread_mutex_t m;
    int done;
} INIT_ONCE;
typedef INIT_ONCE *PINIT_ONCE;
#define INIT_ONCE_STATIC_INIT {PTHREAD_MUTEX_INITIALIZER, 0}
typedef BOOL (*PINIT_ONCE_FN)(PINIT_ONCE, PVOID, PVOID *);
static inline BOOL InitOnceExecuteOnce(INIT_ONCE *o, PINIT_ONCE_FN fn, PVOID param, PVOID *ctx) {
    if (__atomic_load_n(&o->done, __ATOMIC_ACQUIRE)) return TRUE;
    pthread_mutex_lock(&o->m);
    if (!o->done) {
        fn(o, param, ctx);
        __atomic_store_n(&o->done, 1, __ATOMIC_RELEASE);
    }
    pthread_mutex_unlock(&o->m);
    return TRUE;
}

typedef DWORD (*LPTHREAD_START_ROUTINE)(LPVOID);
typedef struct {
    LPTHREAD_START_ROUTINE fn;
    LPVOID arg;
} ShimThreadStart;
static void *shim_thread_main(void *p) {
    ShimThreadStart s = *(ShimThreadStart *)p;
    free(p);
    s.fn(s.arg);
    return NULL;
}
static inline HANDLE CreateThread(void *attr, SIZE_T stack, LPTHREAD_START_ROUTINE fn, LPVOID arg, DWORD flags,
                                  DWORD *tid) {
    (void)attr; (void)stack; (void)flags; (void)tid;
    ShimThreadStart *s = (ShimThreadStart *)malloc(sizeof *s);
    if (!s) return NULL;
    s->fn = fn;
    s->arg = arg;
    pthread_t th;
    if (pthread_create(&th, NULL, shim_thread_main, s) != 0) {
        free(s);
        return NULL;
    }
    pthread_detach(th);
    return (HANDLE)1;
}
static inline BOOL CloseHandle(HANDLE h) { (void)h; return TRUE; }

static inline LONG InterlockedIncrement(volatile LONG *x) { return __atomic_add_fetch(x, 1, __ATOMIC_SEQ_CST); }
static inline LONG InterlockedDecrement(volatile LONG *x) { return __atomic_sub_fetch(x, 1, __ATOMIC_SEQ_CST); }

typedef struct {
    DWORD dwNumberOfProcessors;
} SYSTEM_INFO;
static inline void GetSystemInfo(SYSTEM_INFO *si) {
    const char *env = getenv("FF_CPUS");
    long n = env ? atol(env) : sysconf(_SC_NPROCESSORS_ONLN);
    if (n > 64) n = 64; /* the reference's pool is sized for one 64-CPU processor group */
    si->dwNumberOfProcessors = n > 0 ? (DWORD)n : 1;
}

typedef union {
    int64_t QuadPart;
} LARGE_INTEGER;
static inline BOOL QueryPerformanceFrequency(LARGE_INTEGER *f) {
    f->QuadPart = 1000000000LL;
    return TRUE;
}
static inline BOOL QueryPerformanceCounter(LARGE_INTEGER *c) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return TRUE;
}

#endif
