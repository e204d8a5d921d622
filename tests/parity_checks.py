"""Shared parity checks of the GPU tests (device results against the oracle).

Hazards of the parity plan: H1 closest hits and the GBuffer bit-exact; H2 NEE
light-selection indices bit-exact while the random streams are in sync; H3
reservoir CandidateCount (M) bit-exact; H4 reservoir winner equal except on at
most 1e-4 of the pixels (a ulp-level weight difference from expf/powf can flip
a decision with a tiny margin; reservoir.h:76-125); H5 radiance, WSum and W
within 1e-4 relative on all but 1 % of the pixels.
"""
import numpy as np

RTOL = 1e-4
ATOL = 1e-6
MAX_OUTLIERS = 0.01
MAX_WINNER_FLIPS = 1e-4
GB_FIELDS = ("position", "depth", "normal", "smooth_normal", "albedo", "uv", "dpdu", "dpdv")


def outliers(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    bad = np.abs(a - b) > (ATOL + RTOL * np.maximum(np.abs(a), np.abs(b)))
    return bad.reshape(len(a), -1).any(1).mean()


def check_gbuffer(g, o, idx=None):
    if idx is not None:
        g, o = g[idx], o[idx]
    assert np.array_equal(g["hit"], o["hit"])
    assert np.array_equal(g["prim_id"], o["prim_id"])
    assert np.array_equal(g["tri_id"], o["tri_id"])
    hit = o["hit"] == 1
    for f in GB_FIELDS:
        assert np.array_equal(g[f][hit].view(np.uint32), o[f][hit].view(np.uint32)), f


def reservoir_fields(res):
    """(has_sample, light, wsum, w, m) of the downloaded "__ris_reservoir" planes."""
    e = res[4]
    meta = e[:, 3].view(np.uint32)
    has = (meta & 1).astype(np.int32)
    light = np.where(has == 1, (meta >> 8).astype(np.int64) - 1, -1).astype(np.int32)
    return has, light, e[:, 0], e[:, 1], e[:, 2].view(np.int32)


def check_reservoirs(res, orc_res, idx, label):
    has, light, wsum, w, m = reservoir_fields(res)
    r = orc_res[idx]
    has, light, wsum, w, m = has[idx], light[idx], wsum[idx], w[idx], m[idx]
    assert np.array_equal(m, r["m"]), f"{label}: reservoir CandidateCount (M) must be bit-exact"
    flips = int(((has != r["has_sample"]) | (light != np.where(r["has_sample"] == 1, r["light"], -1))).sum())
    print(f"{label}: winner flips {flips} of {len(m)} pixels")
    assert flips <= max(1, MAX_WINNER_FLIPS * len(m)), f"{label}: reservoir winner differs on {flips} pixels"
    both = (has == 1) & (r["has_sample"] == 1)
    assert both.mean() > 0.2, f"{label}: too few engaged reservoirs to compare"
    f_wsum = outliers(wsum[both], r["wsum"][both])
    f_w = outliers(w[both], r["w"][both])
    print(f"{label}: WSum outliers {f_wsum:.2e}, W outliers {f_w:.2e}")
    assert f_wsum <= MAX_OUTLIERS and f_w <= MAX_OUTLIERS


def check_nee(gpu_lights, trace, hit, n_nee, label):
    gl = gpu_lights.reshape(-1, n_nee)[hit]
    t = trace[hit]
    assert (t["n_nee_idx"] == n_nee).all(), f"{label}: oracle recorded {np.unique(t['n_nee_idx'])} NEE candidates"
    ol = t["nee_light"][:, :n_nee]
    same = (gl == ol).all(1)
    print(f"{label}: NEE light indices equal on {same.mean():.6f} of {len(same)} hit pixels")
    assert same.all(), f"{label}: NEE light-selection indices differ on {(~same).sum()} pixels"
    assert (gl >= 0).mean() > 0.5
