"""torch.autograd wrapper of the radiance estimate, for gradient checks only.

    rad = RadianceEstimate.apply(pos4, pow4, qpos4, qnrm4, k, r_max, filter)

forward builds a photon map from (pos4, pow4) and runs the exact-kNN query
with neighbour lists; backward calls the engine's adjoint (pm_query_backward)
with those lists.  Gradients come back for pos4 (xyz, w = 0) and pow4
(rgb, w = 0).  The engine itself does not depend on autograd.
"""
from __future__ import annotations

import torch

from .photon_map import PhotonMap


class RadianceEstimate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos4, pow4, qpos4, qnrm4, k: int, r_max: float, filt: str = "epanechnikov",
                cone_k: float = 1.0, min_found: int = 0):
        pm = PhotonMap(int(pos4.shape[0]), global_q_radius_max=r_max, knn_target_count=k)
        pm.build(pos4.detach().contiguous(), pow4.detach().contiguous())
        kw = dict(k=k, r_max=r_max, filter=filt, cone_k=cone_k, min_found=min_found)
        out = pm.query(qpos4.contiguous(), qnrm4.contiguous(), want_nbr=True, **kw)
        ctx.pm, ctx.kw, ctx.out = pm, kw, out
        ctx.save_for_backward(qpos4, qnrm4)
        return out["rad"][:, :3].clone()

    @staticmethod
    def backward(ctx, grad_rad):
        qpos4, qnrm4 = ctx.saved_tensors
        gpow, gpos = ctx.pm.query_backward(qpos4.contiguous(), qnrm4.contiguous(), grad_rad.contiguous().float(),
                                           nbr=ctx.out["nbr"], count=ctx.out["count"], **ctx.kw)
        ctx.pm.close()
        return gpos, gpow, None, None, None, None, None, None, None
