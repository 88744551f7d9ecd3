"""Floating-point error of the CUDA path's Jaccard, core and accessory outputs,
stated against the FP64 oracle and against the float-LDLT restatement of the
reference's fit_slope (src/dist/linear_regression.cpp:16-60).

The reference fits log J on k in float (Eigen LDLT on the 2x2 normal
equations).  That solve is itself off the exact least-squares fit, most on
the intercept (accessory), which extrapolates to k = 0: by more than 1e-5 on
about 2% of the pairs of the 4,096-sample workload, up to 1.2e-4.  This build fits in double (within 1e-6 of the
FP64 oracle), and the reference's own golden vectors agree with the double
fit to 1.3e-7 (tests/test_oracle_golden.py).  A pair is called well
conditioned when the float restatement agrees with the FP64 fit to WELL, and
the 1e-5 bar against the float restatement is asserted on those pairs; the
others are counted and reported, and held to the FP64 bar like every pair.
"""
import numpy as np

TOL_F64 = 1e-6     # GPU vs the FP64 oracle, core/accessory
TOL_REF = 1e-5     # GPU vs the float-LDLT restatement, on well-conditioned pairs
WELL = 5e-6        # float restatement vs FP64 fit, both outputs


def report(jac_got, jac_want, ca_got, ca_f64, ca_f32):
    """Per-output error statistics (max, 99.9th percentile, pairs above 1e-5)."""
    out = {"pairs": int(ca_got.shape[0])}
    dj = np.abs(jac_got.astype(np.float64) - jac_want)
    out["jaccard_vs_f64"] = {"max": float(dj.max()) if dj.size else 0.0,
                             "p99.9": float(np.quantile(dj, 0.999)) if dj.size else 0.0}
    d64 = np.abs(ca_got.astype(np.float64) - ca_f64)
    d32 = np.abs(ca_got.astype(np.float64) - ca_f32)
    ref_err = np.abs(ca_f32.astype(np.float64) - ca_f64)
    well = (ref_err <= WELL).all(axis=1)
    for c, name in enumerate(("core", "accessory")):
        out[f"{name}_vs_f64"] = {"max": float(d64[:, c].max()),
                                 "p99.9": float(np.quantile(d64[:, c], 0.999)),
                                 "above_1e-5": int((d64[:, c] > 1e-5).sum())}
        out[f"{name}_vs_f32_ldlt"] = {"max": float(d32[:, c].max()),
                                      "p99.9": float(np.quantile(d32[:, c], 0.999)),
                                      "above_1e-5": int((d32[:, c] > 1e-5).sum()),
                                      "max_well_conditioned": float(d32[well, c].max())
                                      if well.any() else 0.0}
    out["well_conditioned"] = int(well.sum())
    out["ill_conditioned"] = int((~well).sum())
    out["ill_conditioned_f32_vs_f64_max"] = float(ref_err[~well].max()) if (~well).any() else 0.0
    return out, well, d64, d32


def check(jac_got, jac_want, ca_got, ca_f64, ca_f32):
    """Asserts the bars and returns the report; the ill-conditioned pairs are
    counted in it (`ill_conditioned`), not bounded."""
    rep, well, d64, d32 = report(jac_got, jac_want, ca_got, ca_f64, ca_f32)
    np.testing.assert_array_equal(jac_got, jac_want)
    assert d64.max() <= TOL_F64, rep
    assert d32[well].max() <= TOL_REF if well.any() else True, rep
    return rep
