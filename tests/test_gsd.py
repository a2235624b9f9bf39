"""GSD snapshot I/O on the CPU: libpdb200's GSD 2.0 file layer against the file-layer oracle in both
directions, growth of the index and name blocks, append, the frame reader's rules
(src/io/RestartIO.jl:20-447) and the electrostatics settings record
(src/electrostatics/Solver.jl:432-466, src/workflow/Electrostatics.jl:318-360).  No GPU call."""
import importlib.util
import os
import types
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def gsdo():
    spec = importlib.util.spec_from_file_location("pdb200_gsd_oracle", ROOT / "oracle" / "gsd_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def lib(pd):
    pd.build()
    return pd


def hoomd_frame(step, n, D, rng, with_types=True):
    box = np.zeros(6, np.float32)
    box[:D] = 20.0
    pos = np.zeros((n, 3), np.float32)
    pos[:, :D] = rng.uniform(-10, 10, (n, D))
    fr = {"configuration/step": np.array([step], np.uint64), "configuration/dimensions": np.array([D], np.uint8),
          "configuration/box": box, "particles/N": np.array([n], np.uint32), "particles/position": pos,
          "particles/velocity": rng.normal(size=(n, 3)).astype(np.float32)}
    if with_types:
        fr["particles/types"] = np.array([[65, 0], [66, 0]], np.int8)
        fr["particles/typeid"] = (np.arange(n) % 2).astype(np.uint32)
    return fr


def test_library_file_reads_back_through_the_oracle(lib, gsdo, tmp_path):
    rng = np.random.default_rng(1)
    path = tmp_path / "lib.gsd"
    chunks = [{"a/u8": np.arange(5, dtype=np.uint8), "a/i32": rng.integers(-9, 9, (7, 3)).astype(np.int32),
               "a/f64": rng.normal(size=4), "a/u64": np.array([2 ** 40 + 3], np.uint64)},
              {"a/i32": rng.integers(-9, 9, (2, 3)).astype(np.int32), "b/f32": rng.normal(size=(3, 6)).astype(np.float32),
               "a/empty": np.zeros(0, np.float32)}]
    with lib.gsdio.GSDFile(path, "w", application="app", schema="hoomd", schema_version=(1, 4)) as h:
        for fr in chunks:
            for k, v in fr.items():
                h.write_chunk(k, v)
            h.end_frame()
    r = gsdo.Reader(path)
    assert r.header["gsd_version"] == (2, 0) and r.header["schema_version"] == (1, 4)
    assert r.header["application"] == "app" and r.header["schema"] == "hoomd"
    assert r.nframes == 2
    assert r.names[:4] == ["a/u8", "a/i32", "a/f64", "a/u64"]
    for f, fr in enumerate(chunks):
        ids = [e["id"] for e in r.index if e["frame"] == f]
        assert ids == sorted(ids)   # sorted by name id inside a frame
        for k, v in fr.items():
            got = r.chunk(f, k)
            assert got is not None and got.dtype == v.dtype
            np.testing.assert_array_equal(got.reshape(v.shape), v)
    assert r.chunk(1, "a/u8") is None


def test_oracle_file_reads_back_through_the_library(lib, gsdo, tmp_path):
    rng = np.random.default_rng(2)
    frames = [hoomd_frame(10 * k, 9, 3, rng) for k in range(3)]
    frames[1]["log/x"] = rng.normal(size=(4, 3))
    path = tmp_path / "ora.gsd"
    gsdo.write(path, frames, application="oracle")
    with lib.gsdio.GSDFile(path, "r") as h:
        assert h.nframes == 3
        hd = h.header()
        assert hd["gsd_version"] == (2, 0) and hd["application"] == "oracle"
        for f, fr in enumerate(frames):
            assert set(h.frame_names(f)) == set(fr)
            for k, v in fr.items():
                got = h.read(h.find(f, k))
                assert got.dtype == v.dtype
                np.testing.assert_array_equal(got.reshape(v.shape), v)
        assert h.find(0, "log/x") is None and h.latest("log/x", 2) is not None


def test_index_and_name_blocks_grow(lib, gsdo, tmp_path):
    # more than 128 index entries and more than 1024 bytes of names force both blocks to move
    path = tmp_path / "grow.gsd"
    names = [f"log/quantity_with_a_long_name_{k:03d}" for k in range(40)]
    with lib.gsdio.GSDFile(path, "w") as h:
        for f in range(6):
            for k, nm in enumerate(names):
                h.write_chunk(nm, np.array([f * 100 + k], np.float64))
            h.end_frame()
    r = gsdo.Reader(path)
    assert r.nframes == 6 and len(r.index) == 240 and r.names == names
    assert r.header["index_allocated_entries"] >= 240 and r.header["namelist_allocated_entries"] > 1024
    for f in range(6):
        for k, nm in enumerate(names):
            assert r.chunk(f, nm)[0] == f * 100 + k


def test_append_continues_after_the_last_frame(lib, gsdo, tmp_path):
    rng = np.random.default_rng(3)
    path = tmp_path / "append.gsd"
    gsdo.write(path, [hoomd_frame(7, 8, 2, rng)])
    with lib.gsdio.gsd_open(path, append=True) as h:
        assert h.nframes == 1
        fr = hoomd_frame(8, 8, 2, rng)
        for k, v in fr.items():
            h.write_chunk(k, v)
        h.write_chunk("log/new_name", np.array([1.5]))
        h.end_frame()
    r = gsdo.Reader(path)
    assert r.nframes == 2 and r.header["application"] == "oracle"
    assert r.chunk(0, "configuration/step")[0] == 7 and r.chunk(1, "configuration/step")[0] == 8
    assert "log/new_name" in r.names
    # append=False replaces the file
    with lib.gsdio.gsd_open(path, append=False) as h:
        assert h.nframes == 0
    assert gsdo.Reader(path).nframes == 0


def test_chunks_written_after_the_last_frame_are_dropped(lib, gsdo, tmp_path):
    path = tmp_path / "partial.gsd"
    h = lib.gsdio.gsd_open(path)
    h.write_chunk("configuration/step", np.array([1], np.uint64))
    h.end_frame()
    h.write_chunk("configuration/step", np.array([2], np.uint64))
    lib.gsdio.gsd_close(h)
    r = gsdo.Reader(path)
    assert r.nframes == 1 and r.chunk(0, "configuration/step")[0] == 1


def test_file_layer_errors(lib, tmp_path):
    bad = tmp_path / "bad.gsd"
    bad.write_bytes(b"\0" * 300)
    with pytest.raises(lib._native.NativeError, match="magic"):
        lib.gsdio.GSDFile(bad, "r")
    with pytest.raises(lib._native.NativeError, match="cannot open"):
        lib.gsdio.GSDFile(tmp_path / "missing.gsd", "r")
    with lib.gsdio.GSDFile(tmp_path / "e.gsd", "w") as h:
        h.write_chunk("x", np.zeros(2, np.float32))
        with pytest.raises(lib._native.NativeError, match="already in frame"):
            h.write_chunk("x", np.zeros(2, np.float32))
        with pytest.raises(TypeError):
            h.write_chunk("c", np.zeros(2, np.complex64))
    with lib.gsdio.GSDFile(tmp_path / "e.gsd", "r") as h:
        with pytest.raises(lib._native.NativeError, match="open for reading"):
            h.write_chunk("y", np.zeros(1, np.float32))
    short = tmp_path / "short.gsd"
    short.write_bytes(b"\xdf\x65" * 20)
    with pytest.raises(lib._native.NativeError, match="too short"):
        lib.gsdio.GSDFile(short, "r")


def test_read_gsd_frame_rules(lib, gsdo, tmp_path):
    """Chunks absent from a frame are inherited from the closest earlier frame (types, box, N); velocities
    are not (zeros with a warning); ``step`` selects by configuration/step, else the 1-based index."""
    rng = np.random.default_rng(4)
    f0 = hoomd_frame(100, 6, 3, rng)
    f0["particles/diameter"] = np.full(6, 1.5, np.float32)
    f0["particles/charge"] = np.array([1, -1, 1, -1, 1, -1], np.float32)
    f0["particles/property/virial"] = rng.normal(size=(6, 6)).astype(np.float32)
    f0["bonds/N"] = np.array([2], np.uint32)
    f0["bonds/types"] = np.array([[98, 111, 110, 100, 0]], np.int8)
    f0["bonds/typeid"] = np.zeros(2, np.uint32)
    f0["bonds/group"] = np.array([[0, 1], [2, 4]], np.uint32)
    f1 = {"configuration/step": np.array([200], np.uint64),
          "particles/position": rng.uniform(-10, 10, (6, 3)).astype(np.float32)}
    path = tmp_path / "rules.gsd"
    gsdo.write(path, [f0, f1])
    with pytest.warns(UserWarning, match="Velocities missing"):
        fr = lib.read_gsd_frame(path)
    assert fr.step == 200 and fr.N == 6 and fr.D == 3 and fr.box == (20.0, 20.0, 20.0)
    np.testing.assert_array_equal(fr.rx, f1["particles/position"][:, 0])
    assert (fr.vx == 0).all()
    assert fr.types == ["A", "B"] and list(fr.typeid) == [1, 2, 1, 2, 1, 2]
    assert "charge" not in fr.particle_properties     # per-frame properties are not inherited
    assert fr.topology.bonds["N"] == 2 and fr.topology.bonds["tuples"] == [(1, 2), (3, 5)]
    step, rx, ry, rz, vx, vy, vz, typeid, tnames, box, force = fr
    assert step == 200 and force is None and len(fr) == 11
    first = lib.read_gsd_frame(path, step=100)
    assert first.step == 100
    np.testing.assert_array_equal(first.vx, f0["particles/velocity"][:, 0])
    np.testing.assert_allclose(first.particle_properties["diameter"], 1.5)
    np.testing.assert_array_equal(first.particle_properties["charge"], f0["particles/charge"])
    np.testing.assert_array_equal(first.particle_properties["virial"], f0["particles/property/virial"])
    assert "property" not in first.particle_properties   # the virial alias is not repeated
    assert lib.read_gsd_frame(path, step=1).step == 100  # no frame has step 1: the first frame
    with pytest.raises(ValueError, match="not found"):
        lib.read_gsd_frame(path, step=7)


def test_incomplete_last_frame_falls_back(lib, gsdo, tmp_path):
    rng = np.random.default_rng(5)
    f0 = hoomd_frame(1, 4, 2, rng)
    # the last frame's positions are a vector, not an N x 3 matrix: it cannot be read
    broken = {"configuration/step": np.array([2], np.uint64), "particles/position": np.zeros(4, np.float32)}
    path = tmp_path / "broken.gsd"
    gsdo.write(path, [f0, broken])
    with pytest.warns(UserWarning, match="incomplete"):
        fr = lib.read_gsd_frame(path)
    assert fr.step == 1 and fr.D == 2 and fr.rz is None


def fake_solver(influence, **kw):
    spec = types.SimpleNamespace(influence=influence, coulomb_prefactor=14.399645, relative_permittivity=1.0,
                                 real_cutoff=9.0, alpha=0.34705, split_shape=None, window_shape=None, order=5,
                                 alias_order=2, net_charge="error", real_space_modifier="none")
    for k, v in kw.items():
        setattr(spec, k, v)
    return types.SimpleNamespace(spec=spec, mesh=(120, 120, 96))


@pytest.mark.parametrize("influence", ["spme", "p3m_ad", "p3m_ik", "esp", "esp_deconvolution"])
def test_settings_record_round_trip(lib, influence, tmp_path):
    extra = dict(split_shape=21.5, window_shape=14.25, order=8) if influence.startswith("esp") else {}
    if influence == "p3m_ik":
        extra = dict(alias_order=3, net_charge="background", real_space_modifier="potential_shift")
    solver = fake_solver(influence, **extra)
    rec = lib.settings_record(solver)
    assert rec.dtype == np.float64 and len(rec) == 15 and rec[0] == 1.0
    exc = [(1, 2, 0.0), (3, 7, 0.5)]
    path = tmp_path / "settings.gsd"
    with lib.gsd_open(path) as h:
        h.write_chunk("configuration/step", np.array([0], np.uint64))
        h.write_chunk("log/electrostatics/settings", rec)
        h.write_chunk("log/electrostatics/exceptions", lib.exceptions_record(exc).reshape(-1, 3))
        h.end_frame()
        h.write_chunk("configuration/step", np.array([1], np.uint64))
        h.end_frame()
    np.testing.assert_array_equal(lib.read_gsd_log(path, "log/electrostatics/settings"), rec)  # inherited
    f = lib.electrostatics_from_gsd(path)
    spec = lib.electrostatics_spec(f)
    assert spec.influence == influence and tuple(f.mesh) == (120, 120, 96)
    assert f.scaled_pairs == ((1, 2, 0.0), (3, 7, 0.5)) and f.exclusions == "none"
    again = lib.settings_record(types.SimpleNamespace(spec=spec, mesh=tuple(f.mesh)))
    np.testing.assert_array_equal(again, rec)


def test_settings_record_errors(lib, tmp_path):
    with pytest.raises(ValueError, match="Unsupported"):
        lib.electrostatics_from_settings(np.zeros(15))
    rec = lib.settings_record(fake_solver("spme"))
    rec[1] = 9
    with pytest.raises(ValueError, match="method code"):
        lib.electrostatics_from_settings(rec)
    path = tmp_path / "none.gsd"
    with lib.gsd_open(path) as h:
        h.write_chunk("log/x", np.array([1], np.int32))
        h.end_frame()
    assert lib.electrostatics_from_gsd(path) is None
    with pytest.raises(ValueError, match="not Float64"):
        lib.read_gsd_log(path, "log/x")
    with pytest.raises(ValueError, match="out of range"):
        lib.read_gsd_log(path, "log/x", frame=3)


def test_particle_system_from_gsd(lib, gsdo, tmp_path):
    rng = np.random.default_rng(6)
    f0 = hoomd_frame(5, 6, 3, rng)
    f0["particles/mass"] = np.array([1, 2, 1, 2, 1, 2], np.float32)
    f0["particles/charge"] = np.array([1, -1, 1, -1, 1, -1], np.float32)
    f0["bonds/N"] = np.array([1], np.uint32)
    f0["bonds/group"] = np.array([[0, 3]], np.uint32)
    path = tmp_path / "system.gsd"
    gsdo.write(path, [f0])
    s = lib.ParticleSystem.from_gsd(path)
    assert s.n == 6 and s.dim == 3 and s.box == (20.0, 20.0, 20.0) and s.types == ["A", "B"]
    np.testing.assert_array_equal(s.positions, f0["particles/position"].astype(float))
    np.testing.assert_array_equal(s.velocities, f0["particles/velocity"].astype(float))
    np.testing.assert_array_equal(s.masses, f0["particles/mass"])
    np.testing.assert_array_equal(s.charges, f0["particles/charge"])
    assert list(s.typeids) == [1, 2, 1, 2, 1, 2] and s.topology.bonds == [(1, 4)]
    assert s.metadata["step"] == 5


def test_gsd_writer_descriptor(lib):
    w = lib.GSDWriter("x.gsd", every=10, write_start=False)
    assert w.mode == "replace" and w.sync_on_write
    with pytest.raises(ValueError, match="replace or append"):
        lib.GSDWriter("x.gsd", mode="overwrite")
    with pytest.raises(ValueError, match="unwrapped"):
        lib.GSDWriter("x.gsd", write_unwrapped=True)
    with pytest.raises(ValueError, match="positive"):
        lib.GSDWriter("x.gsd", every=0)
