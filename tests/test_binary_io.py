"""Binary CSR files (gsofa_write/read_csr_binary, convert_dat): host-only
round trips and the errors a damaged file must produce, plus (on a GPU) that
a matrix loaded from its binary file factors exactly like the ASCII one."""
import os
import subprocess

import numpy as np
import pytest

from tests.helpers import load_bc, random_pattern, scrambled_csr


def _write_dat(d, beg, end, col, n):
    paths = [os.path.join(d, "%s_%d.dat" % (k, n)) for k in ("colbeg", "colend", "csr")]
    with open(paths[0], "w") as f:
        f.write(" ".join(map(str, beg.tolist())))
    with open(paths[1], "w") as f:
        f.write(" ".join(map(str, end.tolist())))
    with open(paths[2], "w") as f:
        f.write("%d %d\n" % (col.shape[0], n) + " ".join(map(str, col.tolist())))
    return paths


@pytest.mark.parametrize("seed", range(4))
def test_round_trip_of_scrambled_rows(tmp_path, seed):
    from gsofatpds_b200 import read_binary, write_binary
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 300))
    beg, end, col = scrambled_csr(rng, random_pattern(rng, n, 0.05), dup_prob=0.2)
    p = str(tmp_path / "m.gsofacsr")
    write_binary(p, beg, end, col)
    b2, e2, c2 = read_binary(p)
    np.testing.assert_array_equal(b2, beg)
    np.testing.assert_array_equal(e2, end)
    np.testing.assert_array_equal(c2, col)


def test_damaged_files_are_io_errors(tmp_path):
    import ctypes
    from gsofatpds_b200 import GsofaError, read_binary, write_binary
    from gsofatpds_b200 import _lib as C
    z = load_bc()
    p = str(tmp_path / "bc.gsofacsr")
    write_binary(p, z["beg"], z["end"], z["col"])
    raw = open(p, "rb").read()
    L = C.load()
    n, nnz = ctypes.c_int32(), ctypes.c_int64()
    assert L.gsofa_read_csr_binary(p.encode(), ctypes.byref(n), ctypes.byref(nnz), None, None,
                                   None) == C.OK
    assert (n.value, nnz.value) == (z["beg"].shape[0], z["col"].shape[0])
    cases = {"flipped": raw[:1000] + bytes([raw[1000] ^ 1]) + raw[1001:],
             "truncated": raw[:-4], "magic": b"X" + raw[1:]}
    for name, data in cases.items():
        q = str(tmp_path / (name + ".gsofacsr"))
        open(q, "wb").write(data)
        with pytest.raises(GsofaError) as e:
            read_binary(q)
        assert e.value.status == C.ERR_IO, name
    q = str(tmp_path / "version.gsofacsr")
    open(q, "wb").write(raw[:8] + (2).to_bytes(4, "little") + raw[12:])
    with pytest.raises(GsofaError) as e:
        read_binary(q)
    assert e.value.status == C.ERR_UNSUPPORTED
    with pytest.raises(GsofaError):
        read_binary(str(tmp_path / "missing.gsofacsr"))


def test_convert_dat_and_cli(tmp_path):
    from gsofatpds_b200 import _lib as C
    from gsofatpds_b200 import convert_dat, read_binary
    z = load_bc()
    n = z["beg"].shape[0]
    paths = _write_dat(str(tmp_path), z["beg"], z["end"], z["col"], n)
    out = str(tmp_path / "bc.gsofacsr")
    convert_dat(*paths, out)
    b, e, c = read_binary(out)
    np.testing.assert_array_equal(b, z["beg"])
    np.testing.assert_array_equal(e, z["end"])
    np.testing.assert_array_equal(c, z["col"])
    out2 = str(tmp_path / "cli.gsofacsr")
    r = subprocess.run([C.CLI_PATH, "--convert", *paths, out2], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert open(out2, "rb").read() == open(out, "rb").read()


@pytest.mark.gpu
def test_binary_load_factors_like_ascii(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gsofatpds_b200 import Context, convert_dat
    from gsofatpds_b200 import _lib as C
    z = load_bc()
    n = z["beg"].shape[0]
    paths = _write_dat(str(tmp_path), z["beg"], z["end"], z["col"], n)
    out = str(tmp_path / "bc.gsofacsr")
    convert_dat(*paths, out)
    with Context(0) as ctx:
        a = ctx.factor(ctx.load_files(*paths))
        b = ctx.factor(ctx.load_binary(out))
        assert a.counts["fill_count"] == b.counts["fill_count"] == 980136
        assert a.counts["n_supernodes"] == b.counts["n_supernodes"]
        for x, y in zip(a.row_counts().values(), b.row_counts().values()):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(a.lmask(), b.lmask())
    r = subprocess.run([C.CLI_PATH, "--binary", out, "128"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Final Number of fill-ins detected: 980136" in r.stdout


def test_malformed_ascii_dat_files_are_io_errors(tmp_path):
    """The reference's three ASCII files, damaged: too few column ids, a
    non-numeric token, a missing file, too few row starts.  The parser (the
    same one gsofa_load_csr_files uses) reports GSOFA_ERR_IO."""
    from gsofatpds_b200 import GsofaError, convert_dat
    from gsofatpds_b200 import _lib as C
    rng = np.random.default_rng(3)
    n = 40
    beg, end, col = scrambled_csr(rng, random_pattern(rng, n, 0.1))
    out = str(tmp_path / "o.gsofacsr")
    good = _write_dat(str(tmp_path), beg, end, col, n)
    convert_dat(*good, out)  # the undamaged files convert
    cases = {}
    d = tmp_path / "short_csr"
    d.mkdir()
    p = _write_dat(str(d), beg, end, col, n)
    with open(p[2], "w") as f:  # header promises more ids than follow
        f.write("%d %d\n" % (col.shape[0] + 5, n) + " ".join(map(str, col.tolist())))
    cases["short_csr"] = p
    d = tmp_path / "token"
    d.mkdir()
    p = _write_dat(str(d), beg, end, col, n)
    with open(p[0], "w") as f:
        f.write(" ".join(map(str, beg.tolist()[:-1])) + " x7")
    cases["token"] = p
    d = tmp_path / "short_beg"
    d.mkdir()
    p = _write_dat(str(d), beg, end, col, n)
    with open(p[1], "w") as f:
        f.write(" ".join(map(str, end.tolist()[:-3])))
    cases["short_end"] = p
    cases["missing"] = [good[0], good[1], str(tmp_path / "nope.dat")]
    for name, paths in cases.items():
        with pytest.raises(GsofaError) as e:
            convert_dat(*paths, str(tmp_path / ("%s.gsofacsr" % name)))
        assert e.value.status == C.ERR_IO, name
