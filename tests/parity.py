"""Helpers of the GPU parity tests: moving synthetic tables to the device, and
per-output relative errors against the float64 oracle."""
import numpy as np

import radix_b200 as rb

# The 1e-5 relative bound on conics, 2D means, depths and rgb, with a floor of
# 1e-6 x max|x| of each output so that values near zero compare absolutely
TOLERANCE = 1e-5
FLOOR = 1e-6


def to_cuda(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.cuda()


def cuda_table(d):
    return rb.Table.from_dict(d, to=to_cuda)


def host(x):
    if hasattr(x, "cpu"):
        x = x.cpu().numpy()
    return x


def u32(x):
    return host(x).view(np.uint32) if host(x).dtype == np.int32 else host(x)


def rel_errors(gpu, orc, mask):
    """max relative error per output, over the splats both sides draw."""
    out = {}
    for name in ("mean2d", "conic", "depth", "opacity", "rgb"):
        if name not in gpu:
            continue
        g = host(gpu[name]).astype(np.float64)
        o = orc[name]
        sel = mask.reshape(mask.shape + (1,) * (o.ndim - mask.ndim))
        sel = np.broadcast_to(sel, o.shape)
        gv, ov = g[sel], o[sel]
        if ov.size == 0:
            out[name] = 0.0
            continue
        floor = FLOOR * max(np.abs(ov).max(), 1e-30)
        out[name] = float(np.max(np.abs(gv - ov) / np.maximum(np.abs(ov), floor)))
    return out


def compare_projection(gpu, orc, cull_keys=True, tolerance=TOLERANCE):
    """Keys bit-exact (except where an eye's cull decision differs, which is
    counted), visible flags, and every float output within tolerance."""
    g_keys = u32(gpu["keys"])
    gvis = host(gpu["opacity"]) > 0 if "opacity" in gpu else None
    ovis = orc["visible"].astype(bool)
    disagree = int(np.sum(gvis != ovis)) if gvis is not None else 0
    key_mismatch = int(np.sum(g_keys != orc["keys"]))
    errs = rel_errors(gpu, orc, ovis & (gvis if gvis is not None else ovis))
    return dict(cull_disagreements=disagree, key_mismatches=key_mismatch, errors=errs,
                drawn=int(ovis.sum()))
