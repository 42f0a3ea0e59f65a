"""Many independent Brill-Lindquist BSSN evolutions advanced together on one GPU.

Each evolution is a full single-patch grid (its own resolution, masses, positions and
CFL timestep) set up through the C ABI exactly like BSSNGrid; libbssn_b200's batch
object then advances all of them with a fixed number of launches per RK4 stage (group
kernels with one block per 128-point tile over the tiles of every grid) and replays the
step as a captured CUDA graph. The tile shape is chosen by `autotune`, which times each
candidate on the batch itself.

Multi-GPU: evolutions are independent, so they shard across ranks with no collective;
`partition_evolutions` gives the load-balanced split (greedy longest-processing-time by
interior point count).
"""

import ctypes as C
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import lib as L

# (0, 0): each grid gets the 128-point brick (i0 x i1 x i2) that pads its interior least.
PER_GRID = (0, 0)
TILE_SHAPES = [PER_GRID, (32, 4), (64, 2), (16, 8), (128, 1)]


def batching_workload(seed: int = 7, n: int = 64) -> List[Dict]:
    """The batched workload: n evolutions on Spherical grids with Nxx drawn from
    [48..128] x [8..32] x [2..16], masses ~U[0.3,0.7], separations ~U[0.6,1.6] (z = +/-sep/2).

    Nxx2 is drawn among the even values: on a cell-centred phi grid the inner-boundary map
    across the polar axis sends phi to phi + pi, which is a grid point only when Nxx2 is even
    (bcstruct_set_up rejects odd Nxx2 for full 3-D Spherical grids)."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n):
        nxx = (int(rng.integers(48, 129)), int(rng.integers(8, 33)), 2 * int(rng.integers(1, 9)))
        m1, m2 = rng.uniform(0.3, 0.7, 2)
        sep = rng.uniform(0.6, 1.6)
        specs.append(dict(coord="Spherical", Nxx=nxx, grid_physical_size=7.5, BH1_mass=float(m1),
                          BH1_posn_z=float(sep / 2), BH2_mass=float(m2), BH2_posn_z=float(-sep / 2)))
    return specs


def partition_evolutions(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Greedy longest-processing-time partition of evolution indices over `world` ranks."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    bins: List[List[int]] = [[] for _ in range(world)]
    load = [0] * world
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        bins[r].append(i)
        load[r] += sizes[i]
    return [sorted(b) for b in bins]


class BatchedEvolutions:
    def __init__(self, specs: Sequence[Dict], device=None):
        import torch

        from .grid import BSSNGrid

        self.grids = [BSSNGrid(device=device, **s) for s in specs]
        self.lib = L.load()
        self.device = self.grids[0].device
        self.stream = torch.cuda.Stream(self.device)
        self._batch = None
        self.config: Optional[Tuple[int, int]] = None
        n = len(self.grids)
        self._cds = (L.PCD * n)(*[C.pointer(g.cd) for g in self.grids])
        self._gds = (L.PGD * n)(*[C.cast(g.gd, L.PGD) for g in self.grids])

    @property
    def interior_points(self) -> int:
        return sum(g.n_interior for g in self.grids)

    def build(self, tile: Tuple[int, int] = PER_GRID, steps_per_graph: int = 1):
        """Create the batch object and capture its graph: `tile` = (bx, by) with bx*by = 128 for
        one shape for every grid, or PER_GRID for a brick chosen per grid."""
        self.free()
        b = C.c_void_p()
        L.check(self.lib.bssn_b200_batch_create(len(self.grids), self._cds, self._gds, tile[0], tile[1],
                                                steps_per_graph, C.c_void_p(self.stream.cuda_stream), C.byref(b)))
        self._batch = b
        self._steps_per_graph = steps_per_graph
        self.config = tuple(tile)

    def run(self, graph_launches: int) -> None:
        if self._batch is None:
            raise RuntimeError("build() first")
        L.check(self.lib.bssn_b200_batch_run(self._batch, graph_launches))

    def info(self) -> Dict[str, int]:
        nt, no, ni = C.c_int(), C.c_int(), C.c_int()
        kn = C.c_ulonglong()
        L.check(self.lib.bssn_b200_batch_info(self._batch, C.byref(nt), C.byref(no), C.byref(ni), C.byref(kn)))
        pts, padded = C.c_longlong(), C.c_longlong()
        L.check(self.lib.bssn_b200_batch_tile_fill(self._batch, C.byref(pts), C.byref(padded)))
        return {"tiles": nt.value, "outer_points": no.value, "inner_points": ni.value, "kernel_nodes": kn.value,
                "tile_fill": pts.value / max(padded.value, 1)}

    def save_states(self):
        return [g.y_n.clone() for g in self.grids], [(g.cd.time, g.cd.nn) for g in self.grids]

    def restore_states(self, saved) -> None:
        ys, tn = saved
        for g, y, (t, n) in zip(self.grids, ys, tn):
            g.y_n.copy_(y)
            g.cd.time, g.cd.nn = t, n

    def autotune(self, steps: int = 2, tiles: Sequence[Tuple[int, int]] = TILE_SHAPES) -> Dict:
        """Time each tile shape on this batch; keep the fastest. The evolutions' states are
        restored afterwards."""
        import torch

        saved = self.save_states()
        torch.cuda.synchronize()
        results = []
        for tile in tiles:
            self.build(tile=tile, steps_per_graph=1)
            self.run(1)  # warm-up
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(self.stream)
            self.run(steps)
            b.record(self.stream)
            b.synchronize()
            results.append((a.elapsed_time(b) / steps, tile))
        self.restore_states(saved)
        torch.cuda.synchronize()
        results.sort()
        best = results[0]
        self.free()
        return {"ms_per_step": best[0], "tile": best[1],
                "table": [{"ms_per_step": r[0], "tile": r[1]} for r in results]}

    def free(self) -> None:
        if getattr(self, "_batch", None) is not None:
            self.lib.bssn_b200_batch_destroy(self._batch)
            self._batch = None

    def close(self) -> None:
        self.free()
        for g in self.grids:
            g.close()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def time_batch(be: BatchedEvolutions, steps: int) -> float:
    """Device time (ms) of `steps` RK4 steps of the whole batch through the captured graph."""
    import torch

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(be.stream)
    be.run(steps // be._steps_per_graph)
    b.record(be.stream)
    b.synchronize()
    return a.elapsed_time(b)


__all__ = ["BatchedEvolutions", "batching_workload", "partition_evolutions", "time_batch", "TILE_SHAPES", "PER_GRID"]
