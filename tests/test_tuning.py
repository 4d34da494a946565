"""CPU tests of the tuning host logic: the autotuner's file format
(ffg_load_tuning: geometry rows and the cost model), the geometry table's
validity rules, and the committed tuning file itself."""
import os

import numpy as np
import pytest


def test_committed_tuning_file_parses(ff):
    assert os.path.exists(ff.TUNING_PATH)
    rows, mlp = 0, None
    for line in open(ff.TUNING_PATH):
        w = line.split()
        if not w or w[0].startswith("#"):
            continue
        if w[0] == "geometry":
            lg, r3, c, wc = map(int, w[1:])
            # the tuner covers lengths from 2^10; a four-step geometry needs
            # row lengths 2^4..2^13 and columns of at least 4 words
            assert 10 <= lg <= 25 and r3 in (0, 1) and 4 <= c <= 13 and lg - c >= 2 and wc in (8, 16, 32, 64)
            rows += 1
        else:
            assert w[0] == "mlp" and int(w[1]) == ff.MLP_NPARAM
            mlp = np.array([float(v) for v in w[2:]], dtype=np.float32)
    assert rows > 0 and mlp is not None and mlp.size == ff.MLP_NPARAM and np.isfinite(mlp).all()


def test_write_and_load_round_trip(ff, tmp_path):
    p = ff.mlp_init(3)
    path = str(tmp_path / "t.txt")
    ff.write_tuning(path, [(16, 0, 11, 32), (15, 1, 9, 16)], p, comment="test")
    old = (ff.get_geometry(16, 0), ff.get_geometry(15, 1))
    try:
        assert ff.load_tuning(path)
        assert ff.get_geometry(16, 0) == (11, 32)
        assert ff.get_geometry(15, 1) == (9, 16)
    finally:
        ff.set_geometry(16, 0, 0, 0)
        ff.set_geometry(15, 1, 0, 0)
        ff.load_tuning()  # back to the committed table
    assert (ff.get_geometry(16, 0), ff.get_geometry(15, 1)) == old


def test_geometry_rules(ff):
    with pytest.raises(ff.FfgError):
        ff.set_geometry(16, 0, 3, 8)      # rows shorter than 2^4
    with pytest.raises(ff.FfgError):
        ff.set_geometry(16, 0, 15, 8)     # rows longer than 2^13
    with pytest.raises(ff.FfgError):
        ff.set_geometry(16, 0, 10, 12)    # tile width not a power of two
    with pytest.raises(ff.FfgError):
        ff.set_geometry(14, 0, 13, 8)     # columns of 2 rows
    with pytest.raises(ff.FfgError):
        ff.set_geometry(24, 1, 10, 64)    # column tile past shared memory
    # the default rule: c = clamp(lg - 7, 8, 13)
    saved = ff.get_geometry(20, 0)
    try:
        ff.set_geometry(20, 0, 0, 0)
        assert ff.get_geometry(20, 0)[0] == 13
        ff.set_geometry(13, 0, 0, 0)
        assert ff.get_geometry(13, 0)[0] == 8
    finally:
        ff.load_tuning()
    assert ff.get_geometry(20, 0) == saved


def test_bad_tuning_file(ff, tmp_path):
    path = tmp_path / "bad.txt"
    path.write_text("geometry 16 0 11\n")
    with pytest.raises(ff.FfgError):
        ff.load_tuning(str(path))
    path.write_text("mlp 3 1 2 3\n")
    with pytest.raises(ff.FfgError):
        ff.load_tuning(str(path))
    ff.load_tuning()
