"""Device workspace cache: one growing byte buffer per device (torch-owned memory)."""
import torch

_cache = {}


def workspace(device: torch.device, nbytes: int) -> torch.Tensor:
    key = (device.type, device.index)
    buf = _cache.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _cache[key] = buf
    return buf


def release():
    _cache.clear()
