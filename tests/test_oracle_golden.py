"""Pins the CPU oracle against the reference's own golden vectors.

test/ppsketch_ref*.npy (test/test-dists.py:156-203) hold, for 28 genomes and
378 pairs, the raw Jaccard per k, the random-corrected Jaccard per k and the
core/accessory fit.  Their input genomes are not shipped, but the three arrays
constrain each other tightly enough to pin every arithmetic step of the oracle
downstream of calc_intersize:
  * raw Jaccard * 64*s64 is an integer count, and count / (64*s64) in double,
    rounded to float, reproduces the stored raw value exactly;
  * the corrected value is observed_excess(raw, r, 1) rounded to float, with
    r = 0 at k >= 19 and r taken from a 3x3 Monte Carlo table at k = 15;
  * the fit of log J on k over the valid range reproduces core/accessory.
"""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN

S64 = 156
UNION = 64 * S64


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLDEN / "ref_goldens.npz"))


@pytest.mark.parametrize("name", ["unphased", "phased"])
def test_raw_jaccard_is_count_over_bins(gold, name):
    raw = gold[f"{name}_raw_jaccard"]
    counts = np.round(raw.astype(np.float64) * UNION).astype(np.uint32)
    assert counts.max() <= UNION
    rebuilt = np.array([[oracle.jaccard(int(c), S64, 0.0) for c in row] for row in counts],
                       dtype=np.float64).astype(np.float32)
    np.testing.assert_array_equal(rebuilt, raw)


def _corrected(obs, r):
    obs = np.asarray(obs, np.float64)
    r = np.asarray(r, np.float64)
    diff = np.where(obs > r, obs - r, 0.0)
    return (diff * 1 / (1 - r)).astype(np.float32)


def test_random_correction_unphased(gold):
    raw = gold["unphased_raw_jaccard"].astype(np.float64)
    cor = gold["unphased_jaccard"]
    obs = np.round(raw * UNION) / UNION
    # k >= 19: the Monte Carlo table is zero, corrected == observed exactly
    np.testing.assert_array_equal(_corrected(obs[:, 1:], 0.0), cor[:, 1:])
    # k = 15: every pair is explained exactly by one of at most 9 float32 table
    # entries (3 clusters x 3 clusters); find them and check every pair.
    j = cor[:, 0].astype(np.float64)
    ident = obs[:, 0] == 1.0          # identical sketches: J = 1 for any r < 1
    np.testing.assert_array_equal(cor[ident, 0], 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        r0 = np.where(ident, np.nan, (obs[:, 0] - j) / (1 - j))
    groups = np.unique(np.round(r0[~ident], 5))
    assert len(groups) <= 9
    explained = ident.copy()
    table = []
    for g in groups:
        members = np.where(np.round(r0, 5) == g)[0]
        base = np.float32(np.median(r0[members])).view(np.int32)
        cands = (base + np.arange(-4000, 4001, dtype=np.int32)).view(np.float32)
        ok = _corrected(obs[members, 0][None, :], cands[:, None].astype(np.float64)) == \
            cor[members, 0][None, :]
        full = np.where(ok.all(axis=1))[0]
        assert len(full) > 0, f"no single float32 table entry explains group {g}"
        table.append(float(cands[full[len(full) // 2]]))
        explained[members] = True
    assert explained.all()
    assert all(0.0 <= r < 0.01 for r in table)


@pytest.mark.parametrize("name", ["unphased", "phased"])
def test_fit_matches_golden(gold, name):
    J = gold[f"{name}_jaccard"]
    kmers = gold[f"{name}_kmers"]
    ca = gold[f"{name}_coreacc"]
    f64 = np.array([oracle.fit_slope(row, kmers, S64) for row in J], np.float32)
    f32 = np.array([oracle.fit_slope(row, kmers, S64, f32=True) for row in J], np.float32)
    err64 = np.abs(f64 - ca).max(axis=0)
    err32 = np.abs(f32 - ca).max(axis=0)
    # the double-precision fit reproduces the shipped results to ~1 float ulp
    assert err64.max() < 2e-7, err64
    # the float LDLT restatement of the current fit_slope stays within 1e-5
    assert err32.max() < 1e-5, err32


def _expect(x, y):
    slope, icpt = np.polyfit(np.asarray(x, np.float64), np.asarray(y, np.float64), 1)
    return (1 - np.exp(slope) if slope < 0 else 0.0, 1 - np.exp(icpt) if icpt < 0 else 0.0)


def test_fit_range_truncation():
    kmers = np.array([15, 17, 19, 21, 23, 25], np.int32)
    tol = 5.0 / UNION
    good = np.exp(-0.1 - 0.05 * kmers[:4])
    # trailing values at or below tolerance are dropped from the fit
    J = np.array(list(good) + [tol / 2, tol * 0.9], np.float32)
    core, acc = oracle.fit_slope(J, kmers, S64)
    ec, ea = _expect(kmers[:4], np.log(J[:4].astype(np.float64)))
    assert ec > 0 and ea > 0
    assert core == pytest.approx(ec, abs=1e-7) and acc == pytest.approx(ea, abs=1e-7)
    # leading ones too; interior values below tolerance stay inside [first, last]
    J2 = np.array([tol / 4, good[0], tol / 2, good[2], good[3], 0.0], np.float32)
    core2, acc2 = oracle.fit_slope(J2, kmers, S64)
    ec2, ea2 = _expect(kmers[1:5], np.log(J2[1:5].astype(np.float64)))
    assert core2 == pytest.approx(ec2, abs=1e-7) and acc2 == pytest.approx(ea2, abs=1e-7)
    # fewer than two valid points: (0, 0), the reference GPU's result
    assert oracle.fit_slope(np.array([0.5, 0, 0, 0, 0, 0], np.float32), kmers, S64) == (0.0, 0.0)
    assert oracle.fit_slope(np.zeros(6, np.float32), kmers, S64) == (0.0, 0.0)
    # positive slope / intercept clamp to zero distance
    J3 = np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6], np.float32)
    assert oracle.fit_slope(J3, kmers, S64)[0] == 0.0


def test_csrs_known_values():
    # csrs: j = 1 - (1 - 1/(2*4^(k-1)))^L for use_rc; r = j1 j2 / (j1 + j2 - j1 j2)
    L = 2_500_000
    for k in (9, 15, 21, 31):
        mc = 2.0 ** ((k - 1) * 2 + 1)
        jv = 1 - (1 - 1 / mc) ** L
        expect = jv * jv / (2 * jv - jv * jv) if jv > 0 else 0.0  # 1 - 2^-61 == 1.0
        assert oracle.csrs(k, True, L, L) == pytest.approx(expect, rel=1e-12)
    assert oracle.csrs(15, False, 0, 1000) == 0.0
