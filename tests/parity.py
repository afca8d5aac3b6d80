"""Per-path parity between the CUDA kernels and the oracle."""

import numpy as np

# Per-path radiance must agree within this relative error in FP32.
PATH_RTOL = 1e-5
# Paths may diverge where a 1-ulp difference in a transcendental flips a
# branch (roulette, lobe choice, an edge hit); at most this fraction may.
MAX_DIVERGED = 0.01


class PathParity:
    def __init__(self, got, want, rtol=PATH_RTOL):
        got = np.asarray(got, dtype=np.float32)
        want = np.asarray(want, dtype=np.float32)
        self.paths = got.shape[0] * got.shape[1]
        hit_same = got[..., 3] == want[..., 3]
        a = got[..., :3].astype(np.float64)
        b = want[..., :3].astype(np.float64)
        scale = np.maximum(np.abs(a), np.abs(b))
        ok = np.all(np.abs(a - b) <= rtol * scale, axis=-1) & hit_same
        exact = np.all(got == want, axis=-1)
        self.within = float(ok.mean())
        self.exact = float(exact.mean())
        self.diverged = 1.0 - self.within
        rel = np.abs(a - b) / np.maximum(scale, 1e-30)
        self.max_rel_within = float(rel[ok].max()) if ok.any() else 0.0
        self.finite = bool(np.all(np.isfinite(got)))

    def __repr__(self):
        return (f"PathParity(paths={self.paths}, exact={self.exact:.5f}, "
                f"within={self.within:.5f}, diverged={self.diverged:.5f}, "
                f"max_rel_within={self.max_rel_within:.3g})")

    def assert_ok(self, max_diverged=MAX_DIVERGED):
        assert self.finite, "non-finite radiance"
        assert self.diverged <= max_diverged, repr(self)
