"""The library's HDF5 subset (hos_h5_* / hos_b200.h5), on the CPU.

* The reference's only shipped input (Csource/2dpar/initpars.h5 and
  initdata.1.h5, written by h5py) decodes to the values the reference's
  driver reads: 256 x 256, Lx = Ly = 3807.99, g = 9.81, h = 1000, T = 50,
  dtsave = 1, rampflg = 1, Tramp = 200, Hs = 4 std(eta0) = 7.27, bat0 = 0.
  Those files exist only where the reference is checked out; the test is
  skipped elsewhere.
* Files the writer makes read back exactly, and their per-dataset object
  header messages (dataspace, datatype, fill value, layout) have the same
  bytes as those h5py/libhdf5 wrote into the shipped files, addresses aside.
* Bad input is an error with a reason, not a crash.
"""
import os
import struct

import numpy as np
import pytest

from hos_b200 import HosError, h5

from oracle import REFERENCE_SRC as REF  # noqa: E402
shipped = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "initpars.h5")),
                             reason="reference checkout not present")


# ------------------------------------------------------------------ a second,
# independent walk of the structure (test infrastructure): root symbol table
# -> B-tree -> symbol-table nodes -> v1 object header messages
def _messages(path):
    d = open(path, "rb").read()
    assert d[:8] == b"\x89HDF\r\n\x1a\n" and d[8] == 0  # superblock v0
    assert struct.unpack("<Q", d[40:48])[0] == len(d)  # end-of-file address
    bt, heap = struct.unpack("<QQ", d[80:96])
    hsize, _, haddr = struct.unpack("<QQQ", d[heap + 8:heap + 32])
    hd = d[haddr:haddr + hsize]
    used = struct.unpack("<H", d[bt + 6:bt + 8])[0]
    out = {}
    names_in_order = []
    for i in range(used):
        child = struct.unpack("<Q", d[bt + 32 + 16 * i:bt + 40 + 16 * i])[0]
        assert d[child:child + 4] == b"SNOD"
        for k in range(struct.unpack("<H", d[child + 6:child + 8])[0]):
            e = child + 8 + 40 * k
            off, oh = struct.unpack("<QQ", d[e:e + 16])
            name = hd[off:hd.index(b"\0", off)].decode()
            names_in_order.append(name)
            nmsg, _, size = struct.unpack("<HII", d[oh + 2:oh + 12])
            p, msgs = oh + 16, {}
            for _ in range(nmsg):
                t, s, fl = struct.unpack("<HHB", d[p:p + 5])
                msgs[t] = (fl, d[p + 8:p + 8 + s])
                p += 8 + s
            out[name] = msgs
    return out, names_in_order


@shipped
def test_shipped_inputs_decode_to_the_reference_values():
    p = h5.read_params(os.path.join(REF, "initpars.h5"))
    assert (p["Nx"], p["Ny"], p["runsubid"], p["saveflg"], p["rampflg"]) == (256, 256, 1, 1, 1)
    assert p["Lx"] == p["Ly"] and abs(p["Lx"] - 3807.99) < 0.01
    assert (p["g"], p["h"], p["T"], p["dtsave"], p["Tramp"]) == (9.81, 1000.0, 50.0, 1.0, 200.0)
    assert p["Kx0"] == 2 * np.pi / p["Lx"]
    ic = os.path.join(REF, "initdata.1.h5")
    assert sorted(h5.names(ic)) == ["bat0", "eta0", "phi0"]
    eta = h5.read(ic, "eta0")
    assert eta.shape == (256, 256) and abs(4 * eta.std() - 7.27) < 0.01
    assert not h5.read(ic, "bat0").any()
    assert np.isfinite(h5.read(ic, "phi0")).all()


@shipped
def test_writer_matches_the_structure_h5py_wrote(tmp_path):
    ref_msgs, ref_order = _messages(os.path.join(REF, "initpars.h5"))
    p = h5.read_params(os.path.join(REF, "initpars.h5"))
    eta = h5.read(os.path.join(REF, "initdata.1.h5"), "eta0")
    phi = h5.read(os.path.join(REF, "initdata.1.h5"), "phi0")
    h5.write_inputs(tmp_path, eta, phi, p["Lx"], p["Ly"], p["g"], int(p["T"]), p["dtsave"], runsubid=1,
                    saveflg=1, rampflg=1, tramp=int(p["Tramp"]), h=p["h"], kp=int(p["KP"]))
    ours, order = _messages(tmp_path / "initpars.h5")
    assert order == ref_order  # members in name order
    assert set(ours) == set(ref_msgs)
    for name, msgs in ref_msgs.items():
        for t in (0x1, 0x3, 0x5):  # dataspace, datatype, fill value: identical bytes
            assert ours[name][t] == msgs[t], (name, hex(t))
        # layout: same version, class and size; the address differs
        assert ours[name][0x8][1][:2] == msgs[0x8][1][:2] and ours[name][0x8][1][10:18] == msgs[0x8][1][10:18]
    for name in ("eta0", "phi0", "bat0"):
        ref_ic, _ = _messages(os.path.join(REF, "initdata.1.h5"))
        ic, _ = _messages(tmp_path / "initdata.1.h5")
        for t in (0x1, 0x3, 0x5):
            assert ic[name][t] == ref_ic[name][t], (name, hex(t))
    assert np.array_equal(h5.read(tmp_path / "initdata.1.h5", "eta0"), eta)
    assert h5.read_params(tmp_path / "initpars.h5") == p


def test_round_trip_types_and_ranks(tmp_path):
    rng = np.random.default_rng(0)
    data = {
        "scalar_f": 3.25, "scalar_i": np.int64(-7), "vec": rng.standard_normal(17),
        "mat": rng.standard_normal((5, 9)), "ints": np.arange(-6, 6).reshape(3, 4), "f32": rng.standard_normal((4, 4)),
        "empty": np.zeros((0, 3)), "one": np.full((1, 1), 0.2),
    }
    path = tmp_path / "t.h5"
    h5.write(path, data, {"f32": h5.F32})
    assert sorted(h5.names(path)) == sorted(data)
    for k, v in data.items():
        got = h5.read(path, k)
        want = np.asarray(v, dtype=np.float32 if k == "f32" else None).astype(np.float64)
        assert got.shape == np.shape(v) and np.array_equal(got, want), k
    assert h5.info(path, "ints")[1] == h5.I64 and h5.info(path, "f32")[1] == h5.F32
    assert h5.info(path, "mat")[1] == h5.F64


def test_many_datasets_span_several_symbol_table_nodes(tmp_path):
    data = {f"d{i:03d}": np.full((2, 2), float(i)) for i in range(100)}
    path = tmp_path / "many.h5"
    h5.write(path, data)
    _, order = _messages(path)
    assert order == sorted(data)
    for k in ("d000", "d057", "d099"):
        assert h5.read(path, k)[0, 0] == float(int(k[1:]))


def test_snapshot_layout(tmp_path):
    eta = np.arange(12.0).reshape(3, 4)
    h5.write_snapshot(tmp_path / "data0.1.h5", 0.4, 9.81, 10.0, 20.0, eta, -eta, 0 * eta)
    assert sorted(h5.names(tmp_path / "data0.1.h5")) == sorted(["time", "g", "Nx", "Ny", "Lx", "Ly", "eta", "phi",
                                                                 "bat"])
    assert h5.info(tmp_path / "data0.1.h5", "time") == ((1, 1), h5.F64)
    assert h5.read(tmp_path / "data0.1.h5", "Ny")[0, 0] == 4.0
    assert np.array_equal(h5.read(tmp_path / "data0.1.h5", "phi"), -eta)


def test_errors_are_reported(tmp_path):
    with pytest.raises(HosError, match="cannot open"):
        h5.read(tmp_path / "missing.h5", "x")
    path = tmp_path / "a.h5"
    h5.write(path, {"x": np.ones(4)})
    with pytest.raises(HosError, match="no dataset"):
        h5.read(path, "y")
    raw = open(path, "rb").read()
    (tmp_path / "trunc.h5").write_bytes(raw[:200])
    with pytest.raises(HosError):
        h5.read(tmp_path / "trunc.h5", "x")
    (tmp_path / "junk.h5").write_bytes(b"\0" * 4096)
    with pytest.raises(HosError, match="signature"):
        h5.names(tmp_path / "junk.h5")
    with pytest.raises(HosError):
        h5.write(tmp_path / "b.h5", {"a/b": 1.0})
    with pytest.raises(ValueError):
        h5.write(tmp_path / "c.h5", {"cube": np.zeros((2, 2, 2))})


def test_damaged_files_fail_cleanly(tmp_path):
    """Truncated files and flipped metadata bytes give an error or (when the
    damage misses what a read needs) a result, never a crash."""
    rng = np.random.default_rng(5)
    good = tmp_path / "good.h5"
    h5.write(good, {"a": rng.standard_normal((6, 5)), "n": np.int64(3), "s": 2.5})
    raw = bytearray(open(good, "rb").read())
    meta = min(len(raw), 3000)

    def probe(path):
        try:
            for name in h5.names(path):
                h5.read(path, name)
        except (HosError, ValueError, MemoryError):
            pass

    for cut in range(0, len(raw), 41):
        p = tmp_path / "cut.h5"
        p.write_bytes(bytes(raw[:cut]))
        probe(p)
    for trial in range(300):
        bad = bytearray(raw)
        for _ in range(int(rng.integers(1, 4))):
            bad[int(rng.integers(0, meta))] = int(rng.integers(0, 256))
        p = tmp_path / "flip.h5"
        p.write_bytes(bytes(bad))
        probe(p)


def test_run_inputs_round_trip(tmp_path):
    """write_inputs stores what the reference's write_hdf5.py stores, plus the
    optional run settings hos_run reads (/M, /scheme, /dt); read_params gives
    them back as get_params would (all read as double)."""
    rng = np.random.default_rng(9)
    eta, phi = rng.standard_normal((8, 16)), rng.standard_normal((8, 16))
    h5.write_inputs(tmp_path, eta, phi, 100.0, 50.0, 9.81, T=12, dtsave=0.5, runsubid=3, saveflg=2, rampflg=1,
                    tramp=20, order=5, scheme=2, dt=0.05)
    p = h5.read_params(tmp_path / "initpars.h5")
    assert (p["Nx"], p["Ny"], p["runsubid"], p["saveflg"]) == (8, 16, 3, 2)
    assert (p["M"], p["scheme"], p["dt"], p["T"], p["dtsave"]) == (5.0, 2.0, 0.05, 12.0, 0.5)
    assert h5.info(tmp_path / "initpars.h5", "M")[1] == h5.I64 and h5.info(tmp_path / "initpars.h5", "dt")[1] == h5.F64
    assert np.array_equal(h5.read(tmp_path / "initdata.3.h5", "phi0"), phi)
    assert not h5.read(tmp_path / "initdata.3.h5", "bat0").any()
    h5.write_inputs(tmp_path / "plain", eta, phi, 1.0, 1.0, 1.0, T=1, dtsave=1.0)
    assert "M" not in h5.read_params(tmp_path / "plain" / "initpars.h5")


def test_make_inputs_cli(tmp_path):
    from hos_b200 import make_inputs

    assert make_inputs.main([str(tmp_path / "j"), "jonswap", "--n", "32", "--lx", "600", "--kp-index", "4",
                             "--order", "4", "--dt", "0.1", "--T", "2"]) == 0
    p = h5.read_params(tmp_path / "j" / "initpars.h5")
    assert (p["Nx"], p["Ny"], p["Lx"], p["M"], p["dt"], p["T"]) == (32, 32, 600.0, 4.0, 0.1, 2.0)
    eta = h5.read(tmp_path / "j" / "initdata.1.h5", "eta0")
    assert eta.shape == (32, 32) and abs(eta.mean()) < 1e-12 and eta.std() > 0
    assert make_inputs.main([str(tmp_path / "s"), "stokes", "--n", "16", "--ny", "8", "--runsubid", "2"]) == 0
    assert h5.read(tmp_path / "s" / "initdata.2.h5", "phi0").shape == (16, 8)
