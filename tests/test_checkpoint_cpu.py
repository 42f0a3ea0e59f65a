"""Checkpoint file format of the reference (CPU: oracle only, no GPU).

The generated write_checkpoint of a checkpoint-enabled project (oracle variant sph3dck) is run
on the CPU and its file is parsed with this library's description of the format: the
checkpoint commondata layout (bssn_b200_checkpoint_commondata, mirrored by
lib.CheckpointCommondata), params_struct, count, indices and the point-major payload. The
parse must give back the oracle's own state and clock, and read_checkpoint must restore them.
"""

import ctypes as C

import numpy as np
import pytest

from nrpy_b200 import lib as L


def _ref(variant):
    from oracle import ref

    if not ref.available(variant):
        pytest.skip("oracle/_ref not built")
    return ref


def test_checkpoint_commondata_layout():
    ref = _ref("sph3dck")
    lay = ref.struct_layout("sph3dck")
    base = ref.struct_layout("sph3d")
    assert lay["sizeof_commondata"] == C.sizeof(L.CheckpointCommondata)
    assert lay["sizeof_commondata"] == base["sizeof_commondata"] + 8
    assert base["sizeof_commondata"] == C.sizeof(L.CommondataStruct)
    lib = ref._load("sph3dck")
    assert lib.ref_offsetof_commondata_checkpoint_every() == L.CheckpointCommondata.checkpoint_every.offset
    assert L.CheckpointCommondata.checkpoint_every.offset == L.CommondataStruct.convergence_factor.offset
    for f in ("dt", "nn"):
        assert lay[f"offsetof_commondata_{f}"] == getattr(L.CheckpointCommondata, f).offset
    assert lay["sizeof_params"] == C.sizeof(L.ParamsStruct) == base["sizeof_params"]


def parse_checkpoint(path):
    """(commondata, [(params, indices, data[count, NUM_EVOL_GFS])]) of a checkpoint file."""
    raw = path.read_bytes()
    off = C.sizeof(L.CheckpointCommondata)
    cd = L.CheckpointCommondata.from_buffer_copy(raw[:off])
    grids = []
    for _ in range(cd.NUMGRIDS):
        p = L.ParamsStruct.from_buffer_copy(raw[off:off + C.sizeof(L.ParamsStruct)])
        off += C.sizeof(L.ParamsStruct)
        count = int(np.frombuffer(raw, dtype="<i4", count=1, offset=off)[0])
        off += 4
        idx = np.frombuffer(raw, dtype="<i4", count=count, offset=off)
        off += 4 * count
        data = np.frombuffer(raw, dtype="<f8", count=count * L.NUM_EVOL_GFS, offset=off)
        off += 8 * count * L.NUM_EVOL_GFS
        grids.append((p, idx, data.reshape(count, L.NUM_EVOL_GFS)))
    assert off == len(raw)
    return cd, grids


def test_reference_checkpoint_parses_and_restores(tmp_path, monkeypatch):
    ref = _ref("sph3dck")
    monkeypatch.chdir(tmp_path)
    rg = ref.RefGrid("sph3dck", (8, 4, 4), 7.5)
    rg.step(3)
    y = rg.y_n()
    t, nn, dt = rg.time, rg.nn(), rg.dt
    rg.write_checkpoint(t)  # checkpoint_every = time: a checkpoint step
    files = list(tmp_path.glob("checkpoint-conv_factor*.dat"))
    assert [f.name for f in files] == ["checkpoint-conv_factor1.00.dat"]
    cd, grids = parse_checkpoint(files[0])
    assert (cd.time, cd.nn, cd.dt, cd.checkpoint_every, cd.NUMGRIDS) == (t, nn, dt, t, 1)
    p, idx, data = grids[0]
    assert (p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2) == rg.N
    assert np.array_equal(idx, np.arange(rg.ntot))
    assert np.array_equal(data.T.reshape(-1), y)
    # the reference's own restart: overwrite the state, read the file back
    rg.set_y_n(np.zeros_like(y))
    rg.step(1)
    assert rg.read_checkpoint() == 1
    assert np.array_equal(rg.y_n(), y)
    assert (rg.time, rg.nn(), rg.t_0(), rg.nn_0(), rg.checkpoint_every()) == (t, nn, t, nn, t)
    rg.close()


def test_reference_checkpoint_cadence(tmp_path, monkeypatch):
    ref = _ref("sph3dck")
    monkeypatch.chdir(tmp_path)
    rg = ref.RefGrid("sph3dck", (8, 4, 4), 7.5)
    rg.step(3)
    rg.write_checkpoint(rg.time * 1.37)  # not within dt/2 of a multiple
    rg.write_checkpoint(0.0)  # checkpoint_every <= 0: never
    assert not list(tmp_path.glob("checkpoint-*.dat"))
    rg.close()


def test_library_reads_reference_commondata_without_gpu(tmp_path, monkeypatch):
    """bssn_b200_read_checkpoint with griddata = NULL touches no GPU: it reads the commondata
    of a file written by the reference's write_checkpoint; without a file it returns 0."""
    ref = _ref("sph3dck")
    lib = L.load()
    monkeypatch.chdir(tmp_path)
    cd = L.CommondataStruct()
    cd.convergence_factor = 1.0
    every = L.REAL()
    assert lib.bssn_b200_read_checkpoint(C.byref(cd), C.byref(every), None, None) == 0  # no file yet
    assert lib.bssn_b200_read_checkpoint(None, None, None, None) == -1  # BSSN_B200_EINVAL
    rg = ref.RefGrid("sph3dck", (8, 4, 4), 7.5, BH1_mass=0.45, BH2_posn_z=-0.35)
    rg.step(3)
    t, nn, dt = rg.time, rg.nn(), rg.dt
    rg.write_checkpoint(t)
    rg.close()
    assert lib.bssn_b200_read_checkpoint(C.byref(cd), C.byref(every), None, None) == 1
    assert (cd.time, cd.nn, cd.dt, every.value) == (t, nn, dt, t)
    assert (cd.BH1_mass, cd.BH2_posn_z, cd.NUMGRIDS, cd.outer_bc_type) == (0.45, -0.35, 1, b"radiation")
