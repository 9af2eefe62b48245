"""The allocation-free clustering entry point (pxl_clusterize_digis_noalloc).

It serves callers that cannot allocate device memory (device memory owned by another
allocator, or a path that must not block on cudaMalloc/cudaFree): the caller passes device
inputs and outputs and the library keeps its scratch in a fixed device array. Its results
must equal those of the context-based entry point pxl_clusterize_digis (exact integers),
also on a second call, since every call reuses the same scratch. This file is collected last
so that a failure here stops a run only after every other test ran.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


def _noalloc(z, cut):
    import torch

    from pixeltrack import _native
    dev = torch.device("cuda:0")
    n = len(z["id"])
    idt = torch.as_tensor(z["id"].astype(np.int16)).to(dev)
    x = torch.as_tensor(z["x"]).to(dev)
    y = torch.as_tensor(z["y"]).to(dev)
    adc = torch.as_tensor(z["adc"]).to(dev)
    ms = torch.zeros(2001, dtype=torch.int32, device=dev)
    cim = torch.zeros(2000, dtype=torch.int32, device=dev)
    mid = torch.zeros(2000, dtype=torch.int32, device=dev)
    clus = torch.zeros(n, dtype=torch.int32, device=dev)
    ido = torch.zeros(n, dtype=torch.int16, device=dev)
    s = torch.cuda.current_stream(dev)
    rc = _native.lib().pxl_clusterize_digis_noalloc(idt.data_ptr(), x.data_ptr(), y.data_ptr(), adc.data_ptr(), n,
                                                    int(cut), ms.data_ptr(), cim.data_ptr(), mid.data_ptr(),
                                                    clus.data_ptr(), ido.data_ptr(), s.cuda_stream)
    assert rc == 0
    s.synchronize()
    u32 = lambda t: t.cpu().numpy().view(np.uint32)
    return {"module_start": u32(ms), "clus_in_module": u32(cim), "module_id": u32(mid), "clus": clus.cpu().numpy(),
            "id": ido.cpu().numpy().view(np.uint16)}


@pytest.mark.parametrize("cut", [True, False])
def test_noalloc_matches_context_entry_on_two_calls(conditions, cut):
    from pixeltrack import PixelChain, default_params
    with PixelChain(conditions, default_params()) as chain:
        for kn in (3, 0):  # two calls in a row: the second one reuses the first one's scratch
            z = np.load(GOLDEN / f"clustering_kn{kn}.npz")
            ref = chain.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=cut)
            got = _noalloc(z, cut)
            nm = int(ref["module_start"][0])
            assert int(got["module_start"][0]) == nm
            assert np.array_equal(got["module_start"][:nm + 1], ref["module_start"][:nm + 1])
            assert np.array_equal(got["module_id"][:nm], ref["module_id"][:nm])
            assert np.array_equal(got["clus_in_module"], ref["clus_in_module"])
            assert np.array_equal(got["clus"], ref["clus"])
            assert np.array_equal(got["id"], ref["id"])


def test_noalloc_empty_input():
    """n = 0 with null digi pointers: one empty chunk, no module."""
    import torch

    from pixeltrack import _native
    dev = torch.device("cuda:0")
    ms = torch.full((2001,), 7, dtype=torch.int32, device=dev)
    cim = torch.zeros(2000, dtype=torch.int32, device=dev)
    mid = torch.zeros(2000, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream(dev)
    rc = _native.lib().pxl_clusterize_digis_noalloc(None, None, None, None, 0, 1, ms.data_ptr(), cim.data_ptr(),
                                                    mid.data_ptr(), None, None, s.cuda_stream)
    assert rc == 0
    s.synchronize()
    assert int(ms[0]) == 0


def test_noalloc_rejects_oversize():
    from pixeltrack import _native
    rc = _native.lib().pxl_clusterize_digis_noalloc(1, 1, 1, 1, (1 << 20) + 1, 1, 1, 1, 1, 1, 1, None)
    assert rc == -4  # PXL_ERR_CAPACITY, nothing launched
