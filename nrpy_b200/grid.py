"""Host-side driver of one BHaH BSSN grid on a B200, through the C ABI.

Mirrors the set-up sequence of the reference's generated main()
(nrpy/infrastructures/BHaH/main_c.py:125-343): CodeParameter defaults ->
numerical_grid_params_Nxx_dxx_xx -> rfm_precompute -> bcstruct_set_up ->
cfl_limited_timestep -> gridfunction storage -> initial_data, then
MoL_step_forward_in_time per step. Gridfunction storage is owned by torch tensors on the
GPU (device memory and streams only; all arithmetic runs in libbssn_b200).
"""

import ctypes as C
from typing import Dict, Optional, Sequence

import numpy as np
import torch

from . import lib as L


def _ptr(t: torch.Tensor):
    assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    return C.cast(C.c_void_p(t.data_ptr()), L.PR)


class BSSNGrid:
    """One single-patch Spherical, SinhSpherical or SinhCylindrical grid with RK4 storage on the GPU.

    Arguments follow the reference's CodeParameters: ``Nxx`` interior points per
    direction, ``grid_physical_size`` (RMAX for Spherical, AMPL for SinhSpherical),
    ``SINHW`` (SinhSpherical; for SinhCylindrical the width along both rho and z),
    Brill-Lindquist masses / z positions, ``CFL_FACTOR``, ``outer_bc_type``
    ("radiation" or "extrapolation") and ``symmetry_axes`` ("" or "2" for the Spherical
    family; "1" for SinhCylindrical, which is built axisymmetric only).
    """

    def __init__(
        self,
        coord: str = "Spherical",
        Nxx: Sequence[int] = (72, 12, 2),
        grid_physical_size: float = 7.5,
        SINHW: float = 0.2,
        BH1_mass: float = 0.5,
        BH1_posn_z: float = 0.5,
        BH2_mass: float = 0.5,
        BH2_posn_z: float = -0.5,
        CFL_FACTOR: float = 0.5,
        eta: float = 1.0,
        outer_bc_type: str = "radiation",
        symmetry_axes: str = "",
        initial_data: bool = True,
        device: Optional[torch.device] = None,
    ):
        if coord not in L.COORD_HASH:
            raise ValueError(f"CoordSystem {coord!r} not supported; choose from {sorted(L.COORD_HASH)}")
        self.lib = L.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        L.check(self.lib.bssn_b200_set_symmetry_axes(symmetry_axes.encode()))
        self.symmetry_axes = symmetry_axes
        self.coord = coord
        self.cd = L.CommondataStruct()
        self.gd = (L.GriddataStruct * L.MAXNUMGRIDS)()
        self.lib.commondata_struct_set_to_default(C.byref(self.cd))
        self.lib.params_struct_set_to_default(C.byref(self.cd), self.gd)
        cd = self.cd
        cd.BH1_mass, cd.BH1_posn_z, cd.BH2_mass, cd.BH2_posn_z = BH1_mass, BH1_posn_z, BH2_mass, BH2_posn_z
        cd.CFL_FACTOR = CFL_FACTOR
        cd.eta = eta
        cd.outer_bc_type = outer_bc_type.encode()
        cd.NUMGRIDS = 1
        g = self.gd[0]
        p = g.params
        p.CoordSystem_hash = L.COORD_HASH[coord]
        p.grid_physical_size = grid_physical_size
        p.SINHW = SINHW
        p.SINHWRHO = p.SINHWZ = SINHW  # SinhCylindrical: the same width along rho and z
        p.grid_idx = 0
        p.gridname = f"grid_{coord}".encode()
        Nx = (C.c_int * 3)(*Nxx)
        self.lib.numerical_grid_params_Nxx_dxx_xx(C.byref(cd), C.byref(g.params), g.xx, Nx, True)
        self._rfm = L.RfmStruct()
        g.rfmstruct = C.pointer(self._rfm)
        self.lib.rfm_precompute_malloc(C.byref(cd), C.byref(g.params), g.rfmstruct)
        self.lib.rfm_precompute_defines(C.byref(cd), C.byref(g.params), g.rfmstruct, g.xx)
        self.lib.bcstruct_set_up(C.byref(cd), C.byref(g.params), g.xx, C.byref(g.bcstruct))
        cd.dt = 1e30
        self.lib.cfl_limited_timestep(C.byref(cd), C.byref(g.params), g.xx)
        cd.nn = cd.nn_0 = 0
        cd.t_0 = cd.time = 0.0
        self.N = (p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2)
        self.ntot = self.N[0] * self.N[1] * self.N[2]
        self.n_interior = p.Nxx0 * p.Nxx1 * p.Nxx2
        ev = L.NUM_EVOL_GFS * self.ntot
        mk = lambda n: torch.zeros(n, dtype=torch.float64, device=self.device)  # noqa: E731
        self.y_n = mk(ev)
        self.run = mk(ev)
        self.k_odd = mk(ev)
        self.k_even = mk(ev)
        self.aux = mk(L.NUM_AUXEVOL_GFS * self.ntot)
        self.diag = mk(L.NUM_DIAG_GFS * self.ntot)
        gf = g.gridfuncs
        gf.y_n_gfs, gf.y_nplus1_running_total_gfs = _ptr(self.y_n), _ptr(self.run)
        gf.k_odd_gfs, gf.k_even_gfs, gf.auxevol_gfs = _ptr(self.k_odd), _ptr(self.k_even), _ptr(self.aux)
        self._stepper = None
        if initial_data:
            self.lib.initial_data(C.byref(cd), self.gd)

    # ------------------------------------------------------------------ accessors
    @property
    def params(self) -> L.ParamsStruct:
        return self.gd[0].params

    @property
    def dt(self) -> float:
        return self.cd.dt

    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def view(self, t: torch.Tensor, ngfs: Optional[int] = None) -> torch.Tensor:
        n = t.numel() // self.ntot if ngfs is None else ngfs
        return t.view(n, self.N[2], self.N[1], self.N[0])

    def interior(self, t: torch.Tensor) -> torch.Tensor:
        G = L.NGHOSTS
        return self.view(t)[:, G:-G, G:-G, G:-G]

    def device_array(self, ptr, n: int, ctype=C.c_double) -> np.ndarray:
        """Copy n elements of a library-owned device array to a host numpy array."""
        out = np.zeros(n, dtype=np.dtype(ctype))
        if n:
            L.check(self.lib.bssn_b200_memcpy(out.ctypes.data_as(C.c_void_p), C.cast(ptr, C.c_void_p),
                                              out.nbytes, 1))
        return out

    def xx(self) -> Sequence[np.ndarray]:
        return [self.device_array(self.gd[0].xx[d], self.N[d]) for d in range(3)]

    def rfm(self) -> Dict[str, np.ndarray]:
        """Host copies of the rfm precompute arrays: the f0 family over xx0; the second family
        over xx1 (Spherical family: sin(xx1) and derivatives) or, for SinhCylindrical, over xx2
        (z'(xx2) and derivatives, the generated project's f3_of_xx2 arrays)."""
        out = {}
        second = 2 if self.coord == "SinhCylindrical" else 1
        for name, _ in L.RfmStruct._fields_:
            n = self.N[0] if name.startswith("f0") else self.N[second]
            out[name] = self.device_array(getattr(self._rfm, name), n)
        return out

    def bcstruct(self):
        """Host copies of (inner_bc_array, {(gz, dirn): outer list}, bc_info)."""
        bc = self.gd[0].bcstruct
        ni = bc.bc_info.num_inner_boundary_points
        inner = (L.InnerptBcStruct * max(ni, 1))()
        if ni:
            L.check(self.lib.bssn_b200_memcpy(C.cast(inner, C.c_void_p), C.cast(bc.inner_bc_array, C.c_void_p),
                                              C.sizeof(L.InnerptBcStruct) * ni, 1))
        outer = {}
        for gz in range(L.NGHOSTS):
            for d in range(3):
                n = bc.bc_info.num_pure_outer_boundary_points[gz][d]
                arr = (L.OuterptBcStruct * max(n, 1))()
                if n:
                    L.check(self.lib.bssn_b200_memcpy(C.cast(arr, C.c_void_p),
                                                      C.cast(bc.pure_outer_bc_array[d + 3 * gz], C.c_void_p),
                                                      C.sizeof(L.OuterptBcStruct) * n, 1))
                outer[(gz, d)] = arr[:n]
        return inner[:ni], outer, bc.bc_info

    # ------------------------------------------------------------------ operators
    def ricci_eval(self, in_gfs: torch.Tensor, aux: torch.Tensor) -> None:
        g = self.gd[0]
        L.check(self.lib.bssn_b200_ricci_eval(C.byref(g.params), g.rfmstruct, _ptr(in_gfs), _ptr(aux), self.stream))

    def rhs_eval(self, aux: torch.Tensor, in_gfs: torch.Tensor, rhs: torch.Tensor, mixed: bool = False) -> None:
        g = self.gd[0]
        f = self.lib.bssn_b200_rhs_eval_mixed if mixed else self.lib.bssn_b200_rhs_eval
        L.check(f(C.byref(self.cd), C.byref(g.params), g.rfmstruct, _ptr(aux), _ptr(in_gfs), _ptr(rhs), self.stream))

    def apply_bcs_outerradiation_and_inner(self, gfs: torch.Tensor, rhs: torch.Tensor) -> None:
        g = self.gd[0]
        L.check(self.lib.bssn_b200_apply_bcs_outerradiation_and_inner(
            C.byref(self.cd), C.byref(g.params), C.byref(g.bcstruct), g.xx, None, None, _ptr(gfs), _ptr(rhs),
            self.stream))

    def apply_bcs_outerextrap_and_inner(self, gfs: torch.Tensor) -> None:
        g = self.gd[0]
        L.check(self.lib.bssn_b200_apply_bcs_outerextrap_and_inner(C.byref(g.params), C.byref(g.bcstruct),
                                                                   _ptr(gfs), self.stream))

    def apply_bcs_inner_only(self, gfs: torch.Tensor, parity_types: Optional[Sequence[int]] = None) -> None:
        g = self.gd[0]
        n = gfs.numel() // self.ntot
        par = None
        if parity_types is not None:
            par = (C.c_int8 * len(parity_types))(*parity_types)
        L.check(self.lib.bssn_b200_apply_bcs_inner_only(C.byref(g.params), C.byref(g.bcstruct), _ptr(gfs), n,
                                                        par, self.stream))

    def enforce_detgammabar_equals_detgammahat(self, gfs: torch.Tensor) -> None:
        g = self.gd[0]
        L.check(self.lib.bssn_b200_enforce_detgammabar_equals_detgammahat(C.byref(g.params), g.rfmstruct,
                                                                          _ptr(gfs), self.stream))

    def constraints_eval(self, in_gfs: Optional[torch.Tensor] = None, diag: Optional[torch.Tensor] = None):
        """H, M^2, |Lambda| on the interior (Ricci recomputed from in_gfs into the aux buffer)."""
        in_gfs = self.y_n if in_gfs is None else in_gfs
        diag = self.diag if diag is None else diag
        g = self.gd[0]
        self.ricci_eval(in_gfs, self.aux)
        L.check(self.lib.bssn_b200_constraints_eval(C.byref(self.cd), C.byref(g.params), g.rfmstruct, _ptr(in_gfs),
                                                    _ptr(self.aux), _ptr(diag), self.stream))
        return diag

    def constraint_norms(self, in_gfs: Optional[torch.Tensor] = None) -> Dict[str, float]:
        """Volume-weighted L2 norms sqrt(sum f^2 dV) and RMS of H, M^2, |Lambda| over the interior."""
        diag = self.constraints_eval(in_gfs)
        out = (C.c_double * 4)()
        g = self.gd[0]
        L.check(self.lib.bssn_b200_constraint_integrals(C.byref(g.params), g.rfmstruct, _ptr(diag), out,
                                                        self.stream))
        vol = out[3]
        names = ["H", "MSQUARED", "LAMBDA_CONSTRAINT"]
        res = {f"{n}_L2": float(np.sqrt(out[k])) for k, n in enumerate(names)}
        res.update({f"{n}_RMS": float(np.sqrt(out[k] / vol)) if vol > 0 else 0.0 for k, n in enumerate(names)})
        res["volume"] = vol
        return res

    def diagnostics(self, output_every: float, nn: Optional[int] = None, time: Optional[float] = None) -> None:
        """The generated project's diagnostics() on this grid: on output steps (time within dt/2
        of a multiple of output_every) the out0d/out1d/out2d/out3d-integrals files are written to
        the current directory. nn and time default to the grid's step counter and time."""
        cd = self.cd
        if nn is not None:
            cd.nn = int(nn)
        if time is not None:
            cd.time = float(time)
        cd.diagnostics_output_every = float(output_every)
        L.check(self.lib.bssn_b200_diagnostics(C.byref(cd), self.gd, self.stream))

    # ------------------------------------------------------------------ checkpoint / restart
    def write_checkpoint(self, checkpoint_every: float) -> bool:
        """write_checkpoint of a project that registers checkpointing: on checkpoint steps (time
        within dt/2 of a multiple of checkpoint_every > 0) checkpoint-conv_factor%.2f.dat is written
        to the current directory in the reference's format. Returns whether it was written."""
        rc = self.lib.bssn_b200_write_checkpoint(C.byref(self.cd), float(checkpoint_every), self.gd, self.stream)
        if rc < 0:
            L.check(rc)
        return rc == 1

    def read_checkpoint(self) -> Optional[float]:
        """read_checkpoint: restore commondata (time, nn, dt, ...; then t_0 = time, nn_0 = nn) and
        y_n from checkpoint-conv_factor%.2f.dat in the current directory. The grid must have the
        saved size and coordinate system. Returns the file's checkpoint_every, or None when there
        is no checkpoint file."""
        every = L.REAL()
        rc = self.lib.bssn_b200_read_checkpoint(C.byref(self.cd), C.byref(every), self.gd, self.stream)
        if rc < 0:
            L.check(rc)
        self.free_stepper()  # a captured graph bakes in dt
        return every.value if rc == 1 else None

    # ------------------------------------------------------------------ time stepping
    def MoL_step_forward_in_time(self, mode: int = 1, mixed: bool = False, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            L.check(self.lib.bssn_b200_mol_step(C.byref(self.cd), self.gd, mode, int(mixed), self.stream))

    def step_from_host(self, host_in: Sequence[torch.Tensor], host_out: Sequence[torch.Tensor], mode: int = 1,
                       mixed: bool = False, on_step=None, graph: bool = True) -> None:
        """One RK4 step for each host state: host_in[i] (pinned, NUM_EVOL_GFS gridfunctions)
        -> device -> one step -> host_out[i].

        The copies overlap the steps: the state alternates between two device buffers, the
        upload of state i+1 runs on its own stream during step i and the download of state i
        on a third stream during step i+1. Steps run in order on a compute stream that follows
        the current stream (they share the grid's stage buffers). With ``graph`` each step is a
        replay of a CUDA graph of one RK4 step captured for that device buffer (two graphs, kept
        until dt, mode or mixed change); otherwise each step's kernels are launched one by one.
        ``on_step(i, y)`` (optional) is called with the compute stream current after step i
        with the device state. y_n_gfs points at this grid's own y_n again on return."""
        n = len(host_in)
        if len(host_out) != n:
            raise ValueError("host_in and host_out must have the same length")
        if getattr(self, "_y_alt", None) is None:
            self._y_alt = torch.empty_like(self.y_n)
        dev = [self.y_n, self._y_alt]
        caller = torch.cuda.current_stream(self.device)
        if getattr(self, "_host_comp", None) is None:
            self._host_comp = torch.cuda.Stream(self.device)
        comp = self._host_comp
        comp.wait_stream(caller)
        h2d, d2h = torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)
        h2d.wait_stream(comp)
        d2h.wait_stream(comp)
        freed = [None, None]  # event: the last download from buffer k has finished
        gf = self.gd[0].gridfuncs
        graphs = self._host_graphs_for(dev, mode, mixed, comp) if graph else None
        try:
            for i in range(n):
                k = i % 2
                with torch.cuda.stream(h2d):
                    if freed[k] is not None:
                        h2d.wait_event(freed[k])
                    dev[k].copy_(host_in[i], non_blocking=True)
                    loaded = torch.cuda.Event()
                    loaded.record(h2d)
                comp.wait_event(loaded)
                if graphs is not None:
                    L.check(self.lib.bssn_b200_stepper_run(graphs[k], 1))
                else:
                    gf.y_n_gfs = _ptr(dev[k])
                    L.check(self.lib.bssn_b200_mol_step(C.byref(self.cd), self.gd, mode, int(mixed),
                                                        C.c_void_p(comp.cuda_stream)))
                if on_step is not None:
                    with torch.cuda.stream(comp):
                        on_step(i, dev[k])
                stepped = torch.cuda.Event()
                stepped.record(comp)
                with torch.cuda.stream(d2h):
                    d2h.wait_event(stepped)
                    host_out[i].copy_(dev[k], non_blocking=True)
                    done = torch.cuda.Event()
                    done.record(d2h)
                freed[k] = done
        finally:
            gf.y_n_gfs = _ptr(self.y_n)
            comp.wait_stream(h2d)
            comp.wait_stream(d2h)
            caller.wait_stream(comp)

    def _host_graphs_for(self, dev, mode: int, mixed: bool, comp):
        """The two one-step graphs of step_from_host (device buffer 0 and 1), captured on comp."""
        key = (int(mode), bool(mixed), comp.cuda_stream, float(self.cd.dt), dev[0].data_ptr(), dev[1].data_ptr())
        cached = getattr(self, "_host_graphs", None)
        if cached is not None and cached[0] == key:
            return cached[1]
        self._free_host_graphs()
        gf = self.gd[0].gridfuncs
        sts = []
        try:
            for k in (0, 1):
                gf.y_n_gfs = _ptr(dev[k])
                st = C.c_void_p()
                L.check(self.lib.bssn_b200_stepper_create(C.byref(self.cd), self.gd, int(mode), int(mixed), 1,
                                                          C.c_void_p(comp.cuda_stream), C.byref(st)))
                sts.append(st)
        except Exception:
            for st in sts:
                self.lib.bssn_b200_stepper_destroy(st)
            raise
        finally:
            gf.y_n_gfs = _ptr(self.y_n)
        self._host_graphs = (key, sts)
        return sts

    def _free_host_graphs(self) -> None:
        cached = getattr(self, "_host_graphs", None)
        if cached is not None:
            for st in cached[1]:
                self.lib.bssn_b200_stepper_destroy(st)
            self._host_graphs = None

    def make_stepper(self, mode: int = 1, mixed: bool = False, steps_per_graph: int = 1, stream=None):
        """Capture `steps_per_graph` RK4 steps into a CUDA graph bound to this grid's buffers."""
        self.free_stepper()
        st = C.c_void_p()
        s = stream if stream is not None else torch.cuda.Stream(self.device)
        self._stepper_stream = s
        L.check(self.lib.bssn_b200_stepper_create(C.byref(self.cd), self.gd, mode, int(mixed), steps_per_graph,
                                                  C.c_void_p(s.cuda_stream), C.byref(st)))
        self._stepper = st
        self._steps_per_graph = steps_per_graph
        return s

    def run_stepper(self, graph_launches: int) -> None:
        if self._stepper is None:
            raise RuntimeError("make_stepper() first")
        L.check(self.lib.bssn_b200_stepper_run(self._stepper, graph_launches))

    def free_stepper(self) -> None:
        """Release the captured graphs (make_stepper's and step_from_host's)."""
        if getattr(self, "_stepper", None) is not None:
            self.lib.bssn_b200_stepper_destroy(self._stepper)
            self._stepper = None
        self._free_host_graphs()

    def close(self) -> None:
        self.free_stepper()
        g = self.gd[0]
        if getattr(self, "_rfm", None) is not None:
            self.lib.rfm_precompute_free(C.byref(self.cd), C.byref(g.params), g.rfmstruct)
            self.lib.bcstruct_free(C.byref(g.bcstruct))
            self._rfm = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
