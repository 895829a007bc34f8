"""Multi-GPU decomposition of many channels: one process per GPU, channels sharded.

Channels are independent ICEEMDAN problems (each carries its own realizations, stages and
stop tests), so the work splits across ranks with no exchange on the data path: every rank
decomposes its own channels on its own GPU, and the only collectives are the optional gather of
the results to rank 0 and the timing reduction (max over ranks).  The reference decomposes one
channel per call (`iceemdanS`/`iceemdanD`, cudaICEEMDAN.cu:619, :1340); its callers loop over
channels on one GPU.

The sharding is deterministic: channels are assigned longest first to the rank with the least
assigned work (samples x realizations), ties to the lowest rank, so ragged batches balance and
every rank computes the same assignment without communicating.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Sequence, Tuple


def shard(lengths: Sequence[int], world: int) -> List[List[int]]:
    """Channel indices per rank for channels of the given lengths (longest-first greedy)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(lengths[i])
    for lst in out:
        lst.sort()
    return out


def rank_channels(lengths: Sequence[int], rank: int, world: int) -> List[int]:
    """The channels rank `rank` of `world` decomposes."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return shard(lengths, world)[rank]


def realization_block(nr: int, rank: int, world: int) -> Tuple[int, int]:
    """Realizations [r0, r1) of part `rank` when the NR realizations of one channel are split
    over `world` ranks: contiguous blocks in rank order, sizes differing by at most one."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    q, rem = divmod(nr, world)
    r0 = rank * q + min(rank, rem)
    return r0, r0 + q + (1 if rank < rem else 0)


class OrderedEnsemble:
    """The exchanges of one channel whose realizations are split over the ranks of a process
    group (contiguous blocks in rank order, realization_block).

    Within a stage, realizations sift independently except for the lock-step stop test (every
    realization of the channel iterates until all have finished: all_finished, an all-reduce
    MIN of one flag per iteration).  At the end of a CEEMDAN stage the ensemble mean sums
    h0_r - mode_r over the realizations in order; to give the one-GPU result bit for bit the
    sums are not all-reduced (that would change the order of the additions) but passed along
    the ranks: rank k receives the running sums from rank k-1, adds its realizations in order
    and sends them on (recv_partial / send_partial, N doubles per stage), and the last rank's
    sums go to every rank (broadcast_last).  The arrays are numpy arrays or torch tensors on
    the process group's device (CPU tensors for gloo)."""

    def __init__(self, rank: int, world: int, group=None, device=None):
        self.rank, self.world, self.group, self.device = rank, world, group, device

    def _tensor(self, t):
        import numpy as np
        import torch
        if isinstance(t, np.ndarray):
            return torch.from_numpy(t)  # shares the array's memory
        return t

    def all_finished(self, local_all: bool) -> bool:
        if self.world <= 1:
            return bool(local_all)
        import torch
        import torch.distributed as dist
        f = torch.tensor([1 if local_all else 0], dtype=torch.int32, device=self.device)
        dist.all_reduce(f, op=dist.ReduceOp.MIN, group=self.group)
        return bool(f.item())

    def recv_partial(self, t) -> None:
        import torch.distributed as dist
        dist.recv(self._tensor(t), src=self.rank - 1, group=self.group)

    def send_partial(self, t) -> None:
        import torch.distributed as dist
        dist.send(self._tensor(t), dst=self.rank + 1, group=self.group)

    def broadcast_last(self, t) -> None:
        if self.world <= 1:
            return
        import torch.distributed as dist
        dist.broadcast(self._tensor(t), src=self.world - 1, group=self.group)


def max_over_ranks(value: float, world: int, device=None) -> float:
    """Maximum of a per-rank float over all ranks (torch.distributed all-reduce MAX); the
    per-rank value itself when world == 1."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int, device=None) -> float:
    """Sum of a per-rank float over all ranks (torch.distributed all-reduce SUM), e.g. the work
    units of ranks whose shares differ; the per-rank value itself when world == 1."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def decompose_channels(channels: Sequence, decompose: Callable, *, rank: int = 0,
                       world: int = 1, gather: bool = True) -> Optional[Dict[int, object]]:
    """Decompose this rank's share of `channels` with `decompose(channel) -> result`.

    Returns {channel index: result} for this rank's channels, or -- when `gather` is true and
    world > 1 -- the results of every rank on rank 0 (gathered as Python objects) and None on
    the other ranks.  `decompose` is normally a closure over `iceemdan` on this rank's GPU;
    the results should be host arrays when they are gathered.
    """
    lengths = [len(c) for c in channels]
    mine = rank_channels(lengths, rank, world)
    local = {i: decompose(channels[i]) for i in mine}
    if not gather or world <= 1:
        return local
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    merged: Dict[int, object] = {}
    for p in parts:
        merged.update(p)
    return dict(sorted(merged.items()))


def decompose_on_streams(pkg, channels: Sequence, num_noise: int, num_imfs: int, max_iter: int,
                         noise_strength: float, *, streams: int = 4, device=None,
                         seeds: Optional[Sequence[int]] = None, **kwargs) -> List[object]:
    """Decompose several channels on one GPU concurrently: `streams` host threads, each with
    its own CUDA stream, take channels longest first and call `pkg.iceemdan` on their stream
    (the library call releases the GIL and allocates its own workspace per call).  Small
    ensembles leave most SMs idle in the per-spline kernels of a single decomposition; running
    channels side by side fills them.  Returns the IMF tensors in channel order; channel i
    uses noise seed seeds[i] (default 1234 + i), so every result equals the single-call one.
    `channels` are 1-D host arrays or tensors; extra keyword arguments go to `iceemdan`."""
    import threading
    import numpy as np
    import torch
    dev = torch.device("cuda") if device is None else torch.device(device)
    if seeds is None:
        seeds = [1234 + i for i in range(len(channels))]
    order = sorted(range(len(channels)), key=lambda i: (-len(channels[i]), i))
    results: List[object] = [None] * len(channels)
    errors: List[BaseException] = []
    lock = threading.Lock()
    queue = list(order)

    def worker():
        torch.cuda.set_device(dev)
        stream = torch.cuda.Stream(device=dev)
        while True:
            with lock:
                if not queue or errors:
                    return
                i = queue.pop(0)
            try:
                with torch.cuda.stream(stream):
                    c = channels[i]
                    y = (c if isinstance(c, torch.Tensor) else
                         torch.as_tensor(np.asarray(c))).to(dev, non_blocking=False)
                    results[i] = pkg.iceemdan(y, num_noise, num_imfs, max_iter, noise_strength,
                                              seed=int(seeds[i]), stream=stream, **kwargs)
                stream.synchronize()
            except BaseException as exc:  # reported to the caller below
                with lock:
                    errors.append(exc)
                return

    threads = [threading.Thread(target=worker) for _ in range(max(1, min(streams, len(channels))))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return results


def decompose_shared_noise(pkg, channels: Sequence, num_noise: int, num_imfs: int,
                           max_iter: int, noise_strength: float, *, seed: int = 1234,
                           device=None, **kwargs) -> List[object]:
    """Decompose channels of one length with the same noise (the reference's behaviour: every
    call seeds its generator with 1234): the noise phase -- the noise modes and the carries it
    leaves, more than half of a decomposition -- runs once, with the first channel, and the
    other channels start from its state.  Every result equals a full call's bit for bit.
    Returns the IMF tensors in channel order."""
    import numpy as np
    import torch
    if not channels:
        return []
    n = len(channels[0])
    if any(len(c) != n for c in channels):
        raise ValueError("channels must share one length")
    dev = torch.device("cuda") if device is None else torch.device(device)

    def tensor(c):
        return (c if isinstance(c, torch.Tensor) else torch.as_tensor(np.asarray(c))).to(dev)

    first, state = pkg.iceemdan(tensor(channels[0]), num_noise, num_imfs, max_iter,
                                noise_strength, seed=seed, return_noise_state=True, **kwargs)
    out = [first]
    for c in channels[1:]:
        out.append(pkg.iceemdan(tensor(c), num_noise, num_imfs, max_iter, noise_strength,
                                seed=seed, noise_state=state, **kwargs))
    return out


def gradients_on_streams(pkg, signals: Sequence, num_noise: int, num_imfs: int, max_iter: int,
                         noise_strength: float, cotangent, *, streams: int = 4, device=None,
                         seed: int = 1234, noise_state=None, **kwargs) -> List[object]:
    """Reverse pass of several signals of one GPU concurrently: `streams` host threads, each
    with its own CUDA stream, take signals in order and run the taped forward
    (pkg.iceemdan_taped), cotangent(imfs) -> d loss / d imfs and the backward entry on their
    stream.  Returns d loss / d y of each signal (float64 CUDA tensors, signal order); each
    equals the single-stream result bit for bit.  noise_state: optional shared noise-phase
    state for signals of one length (iceemdan(..., return_noise_state=True)).  `signals` are
    1-D float64 CUDA tensors."""
    import threading
    import torch
    dev = torch.device("cuda") if device is None else torch.device(device)
    results: List[object] = [None] * len(signals)
    errors: List[BaseException] = []
    lock = threading.Lock()
    queue = list(range(len(signals)))

    def worker():
        torch.cuda.set_device(dev)
        stream = torch.cuda.Stream(device=dev)
        stream.wait_stream(torch.cuda.current_stream(dev))  # inputs made on the caller's stream
        while True:
            with lock:
                if not queue or errors:
                    return
                i = queue.pop(0)
            try:
                with torch.cuda.stream(stream):
                    imfs, tape = pkg.iceemdan_taped(signals[i], num_noise, num_imfs, max_iter,
                                                    noise_strength, seed=seed, stream=stream,
                                                    noise_state=noise_state, **kwargs)
                    results[i] = tape.backward(cotangent(imfs), stream=stream)
                    tape.free()
                stream.synchronize()
            except BaseException as exc:  # reported to the caller below
                with lock:
                    errors.append(exc)
                return

    threads = [threading.Thread(target=worker) for _ in range(max(1, min(streams, len(signals))))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return results
