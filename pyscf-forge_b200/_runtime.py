"""Device plumbing: streams, pointers, cached workspaces, host<->device
conversion.  torch is used only to own device memory and streams."""
import ctypes

import numpy as np
import torch

from . import _capi

_WORKSPACES = {}


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("pyscf-forge_b200 needs a CUDA device (sm_100a); none is visible")
    _capi.load()


def device():
    require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def workspace(slot, nbytes):
    """A cached device byte buffer per (device, slot); grown on demand.
    Buffers are stream-ordered on the current stream."""
    dev = device()
    key = (dev.index, slot)
    buf = _WORKSPACES.get(key)
    nbytes = max(int(nbytes), 256)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        _WORKSPACES[key] = buf
    return buf


def release_workspaces():
    _WORKSPACES.clear()


def to_dev(x, dtype=torch.float64):
    """numpy / torch -> contiguous device tensor (no copy when already there)."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device(), dtype=dtype)
    else:
        t = torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.float64 if dtype == torch.float64 else None)),
                            device=device())
        if t.dtype != dtype:
            t = t.to(dtype)
    return t.contiguous()


def like_input(result, ref):
    """Return a torch tensor if the caller passed torch, else numpy.  A
    device result for a pinned host input comes back in pinned host memory
    (one DMA copy at link speed)."""
    if isinstance(ref, torch.Tensor):
        if ref.device.type == "cpu" and result.is_cuda and ref.is_pinned():
            out = torch.empty(result.shape, dtype=result.dtype, pin_memory=True)
            out.copy_(result)
            return out
        return result.to(ref.device)
    return result.detach().cpu().numpy()


def eri_pair_matrix(eri, norb):
    """Four-fold (npair, npair) pair matrix from full, 4-fold or 8-fold
    storage (the layout pyscf/lib/mcscf/fci_gas.h:171-176 uses)."""
    norb = int(norb)
    npair = norb * (norb + 1) // 2
    if isinstance(eri, torch.Tensor):
        e = eri.detach().to("cpu", torch.float64).numpy()
    else:
        e = np.asarray(eri, dtype=np.float64)
    if e.size == npair * npair:
        return np.ascontiguousarray(e.reshape(npair, npair))
    if e.size == norb ** 4:
        e = e.reshape(norb, norb, norb, norb)
        i, j = np.tril_indices(norb)
        return np.ascontiguousarray(e[i, j][:, i, j])
    if e.size == npair * (npair + 1) // 2:
        out = np.zeros((npair, npair))
        iu = np.tril_indices(npair)
        out[iu] = e.ravel()
        out = out + out.T - np.diag(np.diag(out))
        return out
    raise ValueError("cannot interpret eri of size %d for norb=%d" % (e.size, norb))
