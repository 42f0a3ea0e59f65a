"""Generate the golden fixtures in tests/golden/ from the reference oracle.

Run in a container where oracle/gen_ref.py has built oracle/_ref (the reference's own
generated BHaH C, compiled). Each case stores a seeded, perturbed input state and the
reference's outputs for it: Ricci_eval, rhs_eval followed by the outer-radiation + inner
BCs, enforce_detgammabar_equals_detgammahat, one full MoL_step_forward_in_time (RK4) from
that state, constraints_eval, plus the grid (xx, dt), the rfm precompute arrays and the
bcstruct maps. Small grids keep the files small; the full-size comparisons run live
against oracle/_ref in the GPU tests.

Usage: python tests/golden/make_golden.py
"""

import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import ref  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent
CASES = {
    # name: (oracle variant, Nxx, grid_physical_size, SINHW, BL masses/positions, seed)
    "sphaxi_16x6x2": ("sphaxi", (16, 6, 2), 7.5, 0.2, (0.5, 0.5, 0.5, -0.5), 11),
    "sph3d_10x6x6": ("sph3d", (10, 6, 6), 7.5, 0.2, (0.45, 0.55, 0.6, -0.4), 12),
    "sinh3d_10x6x6": ("sinh3d", (10, 6, 6), 10.0, 0.2, (0.5, 0.6, 0.4, -0.7), 13),
}


def make(name, variant, Nxx, L, sinhw, bh, seed):
    m1, z1, m2, z2 = bh
    rg = ref.RefGrid(variant, Nxx, L, SINHW=sinhw, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    y0 = rg.y_n()
    inp = ref.perturbed_state(rg, seed=seed)
    ricci = rg.ricci(inp)
    rhs = rg.rhs(ricci, inp)
    rhs_bc = rhs.copy()
    rg.bc_radiation(inp.copy(), rhs_bc)
    enf = inp.copy()
    rg.enforce(enf)
    cons = rg.constraints(inp, ricci)
    rg.set_y_n(inp)
    rg.step(1)
    step1 = rg.y_n()
    inner, outer = rg.bcstruct()
    arrays = dict(
        N=np.array(rg.N), Nxx=np.array(Nxx), grid_physical_size=L, SINHW=sinhw, bh=np.array(bh), seed=seed,
        dt=rg.dt, xx0=rg.xx()[0], xx1=rg.xx()[1], xx2=rg.xx()[2],
        initial_data=y0, input=inp, ricci=ricci, rhs_bc=rhs_bc, enforce_hDD=enf.reshape(24, -1)[11:17].reshape(-1),
        constraints=cons.reshape(-1), step1=step1, dV=rg.dV().reshape(-1),
        inner_dst=inner["dstpt"], inner_src=inner["srcpt"], inner_parity=inner["parity"],
    )
    nf0 = 4 if variant == "sinh3d" else 1
    rf = {}
    if variant == "sinh3d":
        for k, nm in enumerate(["f0_of_xx0", "f0_of_xx0__D0", "f0_of_xx0__DD00", "f0_of_xx0__DDD000"]):
            rf[nm] = rg.rfm_field(k, rg.N[0])
        for k, nm in enumerate(["f1_of_xx1", "f1_of_xx1__D1", "f1_of_xx1__DD11"]):
            rf[nm] = rg.rfm_field(nf0 + k, rg.N[1])
    else:
        rf["f0_of_xx0"] = rg.rfm_field(0, rg.N[0])
        for k, nm in enumerate(["f1_of_xx1", "f1_of_xx1__D1", "f1_of_xx1__DD11"]):
            rf[nm] = rg.rfm_field(1 + k, rg.N[1])
    for nm, a in rf.items():
        arrays["rfm_" + nm] = a
    for (gz, d), o in outer.items():
        arrays[f"outer_{gz}_{d}"] = np.stack([o["i0"], o["i1"], o["i2"], o["FACEX0"], o["FACEX1"], o["FACEX2"]],
                                             axis=-1).astype(np.int16) if len(o) else np.zeros((0, 6), np.int16)
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    rg.close()
    print(name, {k: np.shape(v) for k, v in arrays.items() if np.size(v) > 1})


if __name__ == "__main__":
    for name, args in CASES.items():
        make(name, *args)
