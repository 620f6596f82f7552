"""Helpers of the gradient tests: seeded upstream gradients, the per-splat
loss L_i = sum over eyes and outputs of <upstream, output>, and its central
finite differences through the float64 oracle."""
import numpy as np

import radix_b200 as rb
from oracle import oracle as orc
from radix_b200.synthetic import Mulberry32

OUTS = ("mean2d", "conic", "depth", "opacity", "rgb")
FIELDS = {"centers": 3, "log_scales": 3, "quats": 4, "opacities": 1}


def upstream(n, eyes, seed=1):
    """N(0, 1) upstream gradients of every differentiated output."""
    rng = Mulberry32(seed)
    shapes = {"mean2d": (eyes, n, 2), "conic": (eyes, n, 3), "depth": (eyes, n), "opacity": (eyes, n),
              "rgb": (eyes, n, 3)}
    return {k: rng.normal(int(np.prod(s))).reshape(s) for k, s in shapes.items()}


def losses(d, camera, up, params=None):
    """L_i per splat, and the forward (visibility, rgb) it came from."""
    ref = orc.project([rb.SplatObject(rb.Table.from_dict(d))], camera, params, 32, cull_keys=True)
    L = np.zeros(d["centers"].shape[0])
    for k in OUTS:
        prod = ref[k] * up[k]
        L += prod.reshape(prod.shape[0], prod.shape[1], -1).sum(axis=(0, 2))
    return L, ref


def finite_differences(d, camera, up, h=1e-4, params=None):
    """Central differences of L_i for every input component of every splat.
    Returns {field: [n][k]} and a mask of (splat, field component) pairs whose
    forward changed a cull decision or crossed the rgb clamp (not differentiable)."""
    _, base = losses(d, camera, up, params)
    n = d["centers"].shape[0]
    deg = d["sh_degree"]
    ncol = (1 + ((deg + 1) ** 2 - 1)) * 3
    fd = {"centers": np.zeros((n, 3)), "log_scales": np.zeros((n, 3)), "quats": np.zeros((n, 4)),
          "opacities": np.zeros((n, 1)), "colors": np.zeros((n, ncol))}
    bad = {k: np.zeros(v.shape, dtype=bool) for k, v in fd.items()}
    for field in fd:
        arr = d[field]
        flat = arr.reshape(n, -1)
        for c in range(flat.shape[1]):
            x0 = flat[:, c].astype(np.float64)
            step = h * np.maximum(1.0, np.abs(x0)) if field != "quats" else np.full(n, h)
            plus = (x0 + step).astype(arr.dtype)
            minus = (x0 - step).astype(arr.dtype)
            vals = []
            for v in (plus, minus):
                dd = dict(d)
                m = flat.copy()
                m[:, c] = v
                dd[field] = m.reshape(arr.shape)
                vals.append(losses(dd, camera, up, params))
            (lp, rp), (lm, rm) = vals
            denom = plus.astype(np.float64) - minus.astype(np.float64)
            fd[field][:, c] = (lp - lm) / denom
            changed = ((rp["visible"] != base["visible"]) | (rm["visible"] != base["visible"])).any(axis=0)
            kink = ((rp["rgb"] == 0) != (rm["rgb"] == 0)).any(axis=(0, 2))
            bad[field][:, c] = changed | kink
    fd["opacities"] = fd["opacities"][:, 0]
    bad["opacities"] = bad["opacities"][:, 0]
    return fd, bad


def compare(analytic, fd, bad, rel=1e-4, floor=1e-3):
    """Per field: the fraction of differentiable entries within rel (with a
    floor of floor x max|fd| of the field) and the worst relative error."""
    report = {}
    for k, f in fd.items():
        a = analytic[k].reshape(f.shape)
        ok = ~bad[k]
        scale = np.maximum(np.abs(f), floor * np.abs(f[ok]).max() if ok.any() else 1.0)
        err = np.abs(a - f) / scale
        report[k] = (float((err[ok] <= rel).mean()) if ok.any() else 1.0, float(err[ok].max()) if ok.any() else 0.0,
                     int(ok.sum()))
    return report
