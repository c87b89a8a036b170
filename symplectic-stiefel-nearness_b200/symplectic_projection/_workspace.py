"""Device workspace cache: one growing byte buffer per (device, stream).

Work enqueued on different streams may run concurrently, so each stream gets
its own scratch; the buffer is allocated while that stream is current, which
keeps the caching allocator's reuse stream-ordered.  Torch owns the memory.
"""
import torch

_cache = {}


def workspace(device: torch.device, nbytes: int) -> torch.Tensor:
    stream = torch.cuda.current_stream(device)
    key = (device.index, stream.cuda_stream)
    buf = _cache.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _cache[key] = buf
    return buf


def release():
    _cache.clear()
