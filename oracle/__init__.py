"""CPU oracle of the shoebox integration path: TEST INFRASTRUCTURE, never product code.

A numpy restatement of XPG's integration (`xpg/integrate.py`, `xpg/integrate_kernels.py`, `xpg/shoebox.py`),
written reflection by reflection. Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py`
may import it, and only as the checker (or, for the baseline, as the timed CPU restatement). The product
(`xpg_b200`) never imports it and has no CPU fallback.

Pinning: the restatement is checked against the golden fixtures in `tests/golden/`, which hold the outputs of the
reference's own `integrate()` run on seeded synthetic sweeps (generator script committed beside them).

Arithmetic contract shared with the CUDA kernels (so that masks, counts and every per-pixel quantity agree bit for
bit between the two):
* per-element float32 operations in a fixed order, IEEE round-to-nearest per operation, fused multiply-adds only
  where the reference's CPU torch kernels fuse them (3-vector norms, cross products, the per-pixel dot products);
* transcendental functions (erf, exp, expm1) evaluated in float64 on the float32 argument and rounded once;
* reductions accumulated in float64 and rounded to float32 where the reference holds the result in float32; the
  profile-fit normal equations and the variance tail stay in float64.
"""
