"""Stand-alone broken-line fits on device tensors (pxl_bl_fit of include/pxl.h).

Inputs are CUDA tensors: hits [H, 3] float64 (x, y, z), hits_ge [H, 6] float32
(global covariance per hit, the toGlobal layout of SOARotation.jl:139-147) and
offsets [n+1] int32 (3..8 hits per track). precision 0 = FP64 throughout,
1 = FP32 arithmetic with the band-system LDL^T solve, the parameter transport and the
covariance in FP64.
"""
from __future__ import annotations

import torch

from . import _native
from ._native import check


def workspace(n_tracks: int, device) -> torch.Tensor:
    """Device scratch for the stand-alone fits of n_tracks tracks (reusable across calls)."""
    return torch.empty(int(_native.lib().pxl_fit_workspace_bytes(n_tracks)), dtype=torch.uint8, device=device)


def bl_fit(hits: torch.Tensor, hits_ge: torch.Tensor, offsets: torch.Tensor, b_field: float,
           precision: int = 0, stream: torch.cuda.Stream | None = None,
           ws: torch.Tensor | None = None) -> dict[str, torch.Tensor]:
    if not (hits.is_cuda and hits_ge.is_cuda and offsets.is_cuda):
        raise ValueError("bl_fit takes CUDA tensors")
    hits = hits.contiguous().to(torch.float64)
    hits_ge = hits_ge.contiguous().to(torch.float32)
    offsets = offsets.contiguous().to(torch.int32)
    n = offsets.numel() - 1
    dev = hits.device
    out = {
        "state": torch.empty((n, 5), dtype=torch.float32, device=dev),
        "cov": torch.empty((n, 15), dtype=torch.float32, device=dev),
        "chi2": torch.empty(n, dtype=torch.float32, device=dev),
        "pt": torch.empty(n, dtype=torch.float32, device=dev),
        "eta": torch.empty(n, dtype=torch.float32, device=dev),
        "status": torch.empty(n, dtype=torch.int32, device=dev),
    }
    s = (stream or torch.cuda.current_stream(dev)).cuda_stream
    ws = workspace(n, dev) if ws is None else ws
    check(_native.lib().pxl_bl_fit(hits.data_ptr(), hits_ge.data_ptr(), offsets.data_ptr(), n, float(b_field),
                                   int(precision), out["state"].data_ptr(), out["cov"].data_ptr(),
                                   out["chi2"].data_ptr(), out["pt"].data_ptr(), out["eta"].data_ptr(),
                                   out["status"].data_ptr(), ws.data_ptr(), ws.numel(), s), "pxl_bl_fit")
    return out


def bl_fit_adjoint(hits: torch.Tensor, hits_ge: torch.Tensor, offsets: torch.Tensor, b_field: float,
                   module: torch.Tensor | None = None, module_pos: torch.Tensor | None = None,
                   align: torch.Tensor | None = None, want_align_grad: bool = False,
                   stream: torch.cuda.Stream | None = None) -> dict[str, torch.Tensor]:
    """chi2 per track and d(chi2)/d(hits) (pxl_bl_fit_adjoint); with module ids and module
    centres, the hits are first moved by the per-module alignment align[M, 6] (tx, ty, tz,
    wx, wy, wz), and want_align_grad returns d(sum chi2)/d(align) (float32 and FP64)."""
    if not (hits.is_cuda and hits_ge.is_cuda and offsets.is_cuda):
        raise ValueError("bl_fit_adjoint takes CUDA tensors")
    hits = hits.contiguous().to(torch.float64)
    hits_ge = hits_ge.contiguous().to(torch.float32)
    offsets = offsets.contiguous().to(torch.int32)
    n = offsets.numel() - 1
    dev = hits.device
    nm = 0 if module_pos is None else module_pos.shape[0]
    ptr = lambda t: 0 if t is None else t.data_ptr()
    if module is not None:
        module = module.contiguous().to(torch.int16)
    if module_pos is not None:
        module_pos = module_pos.contiguous().to(torch.float64)
    if align is not None:
        align = align.contiguous().to(torch.float32)
    out = {"chi2": torch.empty(n, dtype=torch.float32, device=dev),
           "grad_hits": torch.empty((hits.shape[0], 3), dtype=torch.float32, device=dev)}
    if want_align_grad:
        out["grad_align"] = torch.empty((nm, 6), dtype=torch.float32, device=dev)
        out["grad_align64"] = torch.empty((nm, 6), dtype=torch.float64, device=dev)
    ws = torch.empty(int(_native.lib().pxl_adjoint_workspace_bytes(n, nm)), dtype=torch.uint8, device=dev)
    s = (stream or torch.cuda.current_stream(dev)).cuda_stream
    check(_native.lib().pxl_bl_fit_adjoint(hits.data_ptr(), hits_ge.data_ptr(), offsets.data_ptr(), n, float(b_field),
                                           ptr(module), ptr(module_pos), ptr(align), nm, out["chi2"].data_ptr(),
                                           out["grad_hits"].data_ptr(), ptr(out.get("grad_align")),
                                           ptr(out.get("grad_align64")), ws.data_ptr(), ws.numel(), s),
          "pxl_bl_fit_adjoint")
    return out


def riemann_fit(hits: torch.Tensor, hits_ge: torch.Tensor, offsets: torch.Tensor, b_field: float,
                precision: int = 0, stream: torch.cuda.Stream | None = None,
                ws: torch.Tensor | None = None) -> dict[str, torch.Tensor]:
    """Riemann helix fits (pxl_riemann_fit): state (n, 5) = (phi, d0, q/pT, cot(theta), zip),
    chi2 (n, 2) = (circle, line), pt, status."""
    if not (hits.is_cuda and hits_ge.is_cuda and offsets.is_cuda):
        raise ValueError("riemann_fit takes CUDA tensors")
    hits = hits.contiguous().to(torch.float64)
    hits_ge = hits_ge.contiguous().to(torch.float32)
    offsets = offsets.contiguous().to(torch.int32)
    n = offsets.numel() - 1
    dev = hits.device
    out = {"state": torch.empty((n, 5), dtype=torch.float32, device=dev),
           "chi2": torch.empty((n, 2), dtype=torch.float32, device=dev),
           "pt": torch.empty(n, dtype=torch.float32, device=dev),
           "status": torch.empty(n, dtype=torch.int32, device=dev)}
    ws = workspace(n, dev) if ws is None else ws
    s = (stream or torch.cuda.current_stream(dev)).cuda_stream
    check(_native.lib().pxl_riemann_fit(hits.data_ptr(), hits_ge.data_ptr(), offsets.data_ptr(), n, float(b_field),
                                        int(precision), out["state"].data_ptr(), out["chi2"].data_ptr(),
                                        out["pt"].data_ptr(), out["status"].data_ptr(), ws.data_ptr(), ws.numel(), s),
          "pxl_riemann_fit")
    return out
