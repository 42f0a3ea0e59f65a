"""Symbolic source of the pointwise algebra: NRPy's own equation modules.

Code-generation time only. The expressions come from the reference's equation modules
(nrpy/equations/general_relativity/BSSN_*.py, nrpy/reference_metric.py); this module
only assembles them into the output lists that each CUDA kernel evaluates, following
how the reference's BHaH generators assemble them:

* ``rhs_exprs``         -- nrpy/infrastructures/BHaH/general_relativity/rhs_eval.py:122-220
  (BSSN_RHSs + 1+log / Gamma-driver gauge RHSs, KO dissipation scaled by ReU[k] and,
  with CAKO, by W = cf), upwind control vector betaU[i] = vetU[i]*ReU[i] (:296-300).
* ``ricci_exprs``       -- Ricci_eval.py:27-167 (BSSN_quantities[...].Ricci_exprs).
* ``constraint_exprs``  -- constraints_eval.py:364-492 (H, M^2, |Lambda constraint|).
* ``enforce_exprs``     -- enforce_detgammabar_equals_detgammahat.py:85-110.

Must be imported with the nrpy package importable; ``symmetry_axes`` is set before any
equation object is built, because nrpy zeroes derivatives across symmetry axes when it
declares them (nrpy/indexedexp.py:598-620).
"""

from typing import Dict, List, Tuple

import sympy as sp

GF_ORDER = [
    "aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22", "alpha", "betU0", "betU1", "betU2",
    "cf", "hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22", "lambdaU0", "lambdaU1",
    "lambdaU2", "trK", "vetU0", "vetU1", "vetU2",
]  # gridfunction index order of the generated BHaH_defines.h (alphabetical)
RBAR_ORDER = ["RbarDD00", "RbarDD01", "RbarDD02", "RbarDD11", "RbarDD12", "RbarDD22"]


def setup_nrpy(symmetry_axes: str, fd_order: int = 4) -> None:
    import nrpy.finite_difference  # noqa: F401  (registers fd_order)
    import nrpy.indexedexp  # noqa: F401  (registers symmetry_axes)
    import nrpy.params as par

    par.set_parval_from_str("Infrastructure", "BHaH")
    par.set_parval_from_str("fp_type", "double")
    par.set_parval_from_str("fd_order", fd_order)
    par.set_parval_from_str("symmetry_axes", symmetry_axes)


def rhs_exprs(coord: str, ko_cako: bool = True) -> Tuple[Dict[str, sp.Expr], List[sp.Expr]]:
    """Return ({rhs name: expr}, betaU) for the 24 evolved gridfunctions."""
    import nrpy.indexedexp as ixp
    import nrpy.reference_metric as refmetric
    from nrpy.equations.general_relativity.BSSN_gauge_RHSs import BSSN_gauge_RHSs
    from nrpy.equations.general_relativity.BSSN_quantities import BSSN_quantities
    from nrpy.equations.general_relativity.BSSN_RHSs import BSSN_RHSs

    key = coord + "_rfm_precompute_RbarDD_gridfunctions"
    rhs = BSSN_RHSs[key]
    alpha_rhs, vet_rhsU, bet_rhsU = BSSN_gauge_RHSs(
        CoordSystem=coord,
        enable_rfm_precompute=True,
        enable_T4munu=False,
        LapseEvolutionOption="OnePlusLog",
        ShiftEvolutionOption="GammaDriving2ndOrder_Covariant",
    )
    d = dict(rhs.BSSN_RHSs_varname_to_expr_dict)
    d["alpha_rhs"] = alpha_rhs
    for i in range(3):
        d[f"vet_rhsU{i}"] = vet_rhsU[i]
        d[f"bet_rhsU{i}"] = bet_rhsU[i]

    Bq = BSSN_quantities[key]
    W = Bq.cf  # EvolvedConformalFactor_cf = "W"
    rfm = refmetric.reference_metric[coord + "_rfm_precompute"]
    ko_gauge = sp.Symbol("KreissOliger_strength_gauge", real=True)
    ko_nongauge = sp.Symbol("KreissOliger_strength_nongauge", real=True)
    if ko_cako:
        ko_gauge *= W
        ko_nongauge *= W
    alpha_dKOD = ixp.declarerank1("alpha_dKOD")
    cf_dKOD = ixp.declarerank1("cf_dKOD")
    trK_dKOD = ixp.declarerank1("trK_dKOD")
    betU_dKOD = ixp.declarerank2("betU_dKOD", symmetry="nosym")
    vetU_dKOD = ixp.declarerank2("vetU_dKOD", symmetry="nosym")
    lambdaU_dKOD = ixp.declarerank2("lambdaU_dKOD", symmetry="nosym")
    aDD_dKOD = ixp.declarerank3("aDD_dKOD", symmetry="sym01")
    hDD_dKOD = ixp.declarerank3("hDD_dKOD", symmetry="sym01")
    for k in range(3):
        d["alpha_rhs"] += ko_gauge * alpha_dKOD[k] * rfm.ReU[k]
        d["cf_rhs"] += ko_nongauge * cf_dKOD[k] * rfm.ReU[k]
        d["trK_rhs"] += ko_nongauge * trK_dKOD[k] * rfm.ReU[k]
        for i in range(3):
            d[f"bet_rhsU{i}"] += ko_gauge * betU_dKOD[i][k] * rfm.ReU[k]
            d[f"vet_rhsU{i}"] += ko_gauge * vetU_dKOD[i][k] * rfm.ReU[k]
            d[f"lambda_rhsU{i}"] += ko_nongauge * lambdaU_dKOD[i][k] * rfm.ReU[k]
            for j in range(i, 3):
                d[f"a_rhsDD{i}{j}"] += ko_nongauge * aDD_dKOD[i][j][k] * rfm.ReU[k]
                d[f"h_rhsDD{i}{j}"] += ko_nongauge * hDD_dKOD[i][j][k] * rfm.ReU[k]

    vetU = ixp.declarerank1("vetU")
    betaU = [vetU[i] * rfm.ReU[i] for i in range(3)]
    # Order the outputs by the evolved gridfunction index.
    name_of = {
        "alpha": "alpha_rhs", "cf": "cf_rhs", "trK": "trK_rhs",
    }
    out: Dict[str, sp.Expr] = {}
    for gf in GF_ORDER:
        if gf in name_of:
            rn = name_of[gf]
        elif gf.startswith("aDD"):
            rn = "a_rhsDD" + gf[3:]
        elif gf.startswith("hDD"):
            rn = "h_rhsDD" + gf[3:]
        elif gf.startswith("lambdaU"):
            rn = "lambda_rhsU" + gf[7:]
        elif gf.startswith("vetU"):
            rn = "vet_rhsU" + gf[4:]
        elif gf.startswith("betU"):
            rn = "bet_rhsU" + gf[4:]
        else:
            raise KeyError(gf)
        out[gf] = d[rn]
    return out, betaU


def ricci_exprs(coord: str) -> Dict[str, sp.Expr]:
    from nrpy.equations.general_relativity.BSSN_quantities import BSSN_quantities

    Bq = BSSN_quantities[coord + "_rfm_precompute"]
    return dict(zip(Bq.Ricci_varnames, Bq.Ricci_exprs))


def constraint_exprs(coord: str) -> Dict[str, sp.Expr]:
    from nrpy.equations.general_relativity.BSSN_constraints import BSSN_constraints

    Bcon = BSSN_constraints[coord + "_rfm_precompute_RbarDD_gridfunctions"]
    return {
        "H": Bcon.H,
        "MSQUARED": Bcon.Msquared,
        "LAMBDA_CONSTRAINT": Bcon.LambdaConstraintMagnitude,
    }


def enforce_exprs(coord: str) -> Dict[str, sp.Expr]:
    import nrpy.indexedexp as ixp
    import nrpy.reference_metric as refmetric
    from nrpy.equations.general_relativity.BSSN_quantities import BSSN_quantities

    Bq = BSSN_quantities[coord + "_rfm_precompute"]
    rfm = refmetric.reference_metric[coord + "_rfm_precompute"]
    _, detgammabar = ixp.symm_matrix_inverter3x3(Bq.gammabarDD)
    absf = sp.Function("nrpyAbs")
    out = {}
    for i in range(3):
        for j in range(i, 3):
            out[f"hDD{i}{j}"] = (absf(rfm.detgammahat) / detgammabar) ** sp.Rational(1, 3) * (
                (rfm.ghatDD[i][j] / rfm.ReDD[i][j]) + Bq.hDD[i][j]
            ) - (rfm.ghatDD[i][j] / rfm.ReDD[i][j])
    return out


def lambda_id_exprs(coord: str) -> Dict[str, sp.Expr]:
    """lambda^i = Lambdabar^i / ReU[i], Lambdabar^i = gammabar^jk (Gammabar^i_jk - Gammahat^i_jk).

    ADM_Initial_Data_Reader__BSSN_Converter.py:462-580 (the reference evaluates it with the
    closed-form reference metric; here the rfm-precompute form of the same quantities).
    """
    import nrpy.reference_metric as refmetric
    from nrpy.equations.general_relativity.BSSN_quantities import BSSN_quantities

    Bq = BSSN_quantities[coord + "_rfm_precompute"]
    rfm = refmetric.reference_metric[coord + "_rfm_precompute"]
    out = {}
    for i in range(3):
        lam = sp.sympify(0)
        for j in range(3):
            for k in range(3):
                lam += Bq.gammabarUU[j][k] * (Bq.GammabarUDD[i][j][k] - rfm.GammahatUDD[i][j][k])
        out[f"lambdaU{i}"] = lam / rfm.ReU[i]
    return out
