"""Checkpoint / restart against the reference's generated write_checkpoint / read_checkpoint (B200).

The reference side is the oracle variant sph3dck: the two_blackholes_collide-style project that
also registers checkpointing (checkpointing.py:473-490). Each direction is checked:
- a checkpoint written by this library is read by the reference's read_checkpoint, and one
  written by the reference's write_checkpoint is read by this library: the restored state is
  bit-identical and the clock (time, nn, dt, t_0 = time, nn_0 = nn) and cadence agree;
- for the same state and clock both writers produce the same params, count, indices and
  payload bytes;
- a run restarted from a checkpoint continues bit-identically to an uninterrupted run;
- the cadence rule, a missing file, a commondata-only read and a grid-size mismatch behave as the
  reference's functions (except that errors return a status instead of exiting).
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NXX = (24, 8, 8)
GPS = 7.5
BH = dict(BH1_mass=0.45, BH1_posn_z=0.4, BH2_mass=0.55, BH2_posn_z=-0.35)
FNAME = "checkpoint-conv_factor1.00.dat"


def _ref():
    from oracle import ref

    if not ref.available("sph3dck"):
        pytest.skip("oracle/_ref not built")
    return ref


def _grid(**kw):
    from nrpy_b200.grid import BSSNGrid

    return BSSNGrid("Spherical", NXX, grid_physical_size=GPS, **BH, **kw)


def _host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_reference_reads_our_checkpoint(cuda, tmp_path, monkeypatch):
    ref = _ref()
    monkeypatch.chdir(tmp_path)
    g = _grid()
    g.MoL_step_forward_in_time(nsteps=4)
    y = _host(g.y_n)
    t, nn, dt = g.cd.time, g.cd.nn, g.cd.dt
    assert nn == 4
    assert g.write_checkpoint(t)
    rg = ref.RefGrid("sph3dck", NXX, GPS, **BH)
    assert rg.dt == dt
    assert rg.read_checkpoint() == 1
    assert np.array_equal(rg.y_n(), y)
    assert (rg.time, rg.nn(), rg.t_0(), rg.nn_0(), rg.checkpoint_every()) == (t, nn, t, nn, t)
    rg.close()
    g.close()


def test_we_read_reference_checkpoint(cuda, tmp_path, monkeypatch):
    import torch

    ref = _ref()
    monkeypatch.chdir(tmp_path)
    rg = ref.RefGrid("sph3dck", NXX, GPS, **BH)
    rg.step(4)
    y = rg.y_n()
    t, nn, dt = rg.time, rg.nn(), rg.dt
    rg.write_checkpoint(1.37 * t)  # not a checkpoint step: nothing written
    assert not (tmp_path / FNAME).exists()
    rg.write_checkpoint(t)
    rg.close()
    g = _grid()
    g.y_n.fill_(0.0)
    g.cd.time, g.cd.nn, g.cd.dt = 0.0, 0, 1.0
    assert g.read_checkpoint() == t
    assert np.array_equal(_host(g.y_n), y)
    assert (g.cd.time, g.cd.nn, g.cd.dt, g.cd.t_0, g.cd.nn_0) == (t, nn, dt, t, nn)
    assert g.cd.NUMGRIDS == 1 and g.cd.outer_bc_type == b"radiation"
    assert (g.cd.BH1_mass, g.cd.BH2_posn_z) == (BH["BH1_mass"], BH["BH2_posn_z"])
    torch.cuda.synchronize()
    g.close()


def test_same_payload_bytes_as_reference(cuda, tmp_path, monkeypatch):
    import torch

    from nrpy_b200 import lib as L

    ref = _ref()
    rg = ref.RefGrid("sph3dck", NXX, GPS, **BH)
    state = ref.perturbed_state(rg, seed=7)
    rg.set_y_n(state)
    g = _grid()
    g.y_n.copy_(torch.from_numpy(state))
    nn, t = 5, 5 * rg.dt
    assert g.cd.dt == rg.dt
    rg.set_clock(nn, t)
    # the same CodeParameters and clock on both sides (the project's defaults, e.g. t_final =
    # grid_physical_size, are its own)
    src = L.CheckpointCommondata.from_buffer_copy(rg.commondata_bytes())
    for name, _ in L.CommondataStruct._fields_:
        setattr(g.cd, name, getattr(src, name))
    for d, writer in (("ref", lambda: rg.write_checkpoint(t)), ("ours", lambda: g.write_checkpoint(t))):
        (tmp_path / d).mkdir()
        monkeypatch.chdir(tmp_path / d)
        writer()
    torch.cuda.synchronize()
    rg.close()
    g.close()
    a = (tmp_path / "ref" / FNAME).read_bytes()
    b = (tmp_path / "ours" / FNAME).read_bytes()
    assert len(a) == len(b)
    hdr = C.sizeof(L.CheckpointCommondata)
    ca = L.CheckpointCommondata.from_buffer_copy(a[:hdr])
    cb = L.CheckpointCommondata.from_buffer_copy(b[:hdr])
    for name, _ in L.CheckpointCommondata._fields_:
        if name != "start_wallclock_time":
            va, vb = getattr(ca, name), getattr(cb, name)
            assert (bytes(va) if hasattr(va, "_length_") else va) == (bytes(vb) if hasattr(vb, "_length_") else vb), name
    pend = hdr + C.sizeof(L.ParamsStruct)
    pa = L.ParamsStruct.from_buffer_copy(a[hdr:pend])
    pb = L.ParamsStruct.from_buffer_copy(b[hdr:pend])
    for name, _ in L.ParamsStruct._fields_:
        va, vb = getattr(pa, name), getattr(pb, name)
        if isinstance(va, float):
            assert va == pytest.approx(vb, rel=1e-14, abs=1e-300), name
        else:
            assert va == vb, name
    assert a[pend:] == b[pend:]  # count, indices and the point-major payload


def test_restart_continues_bitwise(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    a = _grid()
    a.MoL_step_forward_in_time(nsteps=6)
    ya = _host(a.y_n)
    b = _grid()
    b.MoL_step_forward_in_time(nsteps=3)
    assert b.write_checkpoint(b.cd.time)
    c = _grid(initial_data=False)
    assert c.read_checkpoint() is not None
    c.MoL_step_forward_in_time(nsteps=3)
    assert np.array_equal(_host(c.y_n), ya)
    assert (c.cd.nn, c.cd.time) == (a.cd.nn, a.cd.time)
    for g in (a, b, c):
        g.close()


def test_cadence_missing_file_and_mismatch(cuda, tmp_path, monkeypatch):
    from nrpy_b200 import lib as L
    from nrpy_b200.grid import BSSNGrid

    monkeypatch.chdir(tmp_path)
    g = _grid()
    assert g.read_checkpoint() is None  # no file yet: a fresh start
    g.MoL_step_forward_in_time(nsteps=3)
    assert not g.write_checkpoint(0.0)
    assert not g.write_checkpoint(-1.0)
    assert not g.write_checkpoint(g.cd.time * 1.37)
    assert not (tmp_path / FNAME).exists()
    assert g.write_checkpoint(g.cd.time)
    # commondata only (griddata NULL), as a driver does before rebuilding its grids
    cd = L.CommondataStruct()
    every = L.REAL()
    cd.convergence_factor = 1.0
    assert g.lib.bssn_b200_read_checkpoint(C.byref(cd), C.byref(every), None, None) == 1
    assert (cd.nn, cd.time, every.value) == (3, g.cd.time, g.cd.time)
    # a grid of another size is refused, and its state and clock are left alone
    h = BSSNGrid("Spherical", (16, 8, 8), grid_physical_size=GPS, **BH)
    before = _host(h.y_n)
    with pytest.raises(L.BssnError, match="mismatch"):
        h.read_checkpoint()
    assert np.array_equal(_host(h.y_n), before) and h.cd.nn == 0
    for x in (g, h):
        x.close()
