"""Transports for a decomposed domain: the two callbacks of kfvm_set_exchange.

The reference runs one block per MPI rank and moves the halo cells and the
boundary face states of every block face shared with another rank by
point-to-point messages, and its step scalars by MPI_Allreduce
(src/LayoutMPI.H:44-97, src/Solver.cpp:345-409, 532-552, 826-1460).  Here the
solver packs those regions into device buffers and hands them to a transport:

* DistExchange -- one rank per process over torch.distributed: NCCL over
  NVLink for device buffers (one rank per GPU), gloo for the host buffers of
  the CPU restatement.  Halo and face messages go through batch_isend_irecv;
  the scalars through all_reduce.
* LocalExchange -- several blocks driven by host threads of one process (one
  endpoint per block), through a mailbox and a barrier with a time limit.  It
  lets one GPU run the blocks of a decomposed domain side by side; no kernel
  ever waits on another block's kernels, only the host threads meet.

Message pairing: in an exchange call every rank sends its low-side buffer to the
rank across its low face and its high-side buffer to the rank across its high
face; the low neighbour's high-side buffer arrives in recv_lo and the high
neighbour's low-side buffer in recv_hi.  With two blocks on a periodic axis both
neighbours are the same rank, so the sends are posted low then high and the
receives high then low (matched in order, as NCCL matches them) and tagged with
the side they were sent from (as gloo matches them).
"""
import ctypes as C
import threading

import kfvm_abi as abi

_SIDE_LO, _SIDE_HI = 0, 1


class _CudaBytes:
    """A device byte range in the CUDA array interface, for torch.as_tensor."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def _view(ptr, nbytes, device):
    """A uint8 tensor over the callback's buffer (no copy)."""
    import torch
    if device is None:
        return torch.frombuffer((C.c_char * int(nbytes)).from_address(int(ptr)), dtype=torch.uint8)
    return torch.as_tensor(_CudaBytes(ptr, nbytes), device=device)


class _Callbacks:
    """Wraps exchange(axis, send_lo, recv_lo, send_hi, recv_hi, nlo, nhi) and
    allreduce(op, values) into the C callbacks; an exception becomes a nonzero
    return, which the solver turns into an error of the step."""

    def __init__(self):
        self.error = None

        def ex(user, axis, send_lo, recv_lo, send_hi, recv_hi, nlo, nhi):
            try:
                self.exchange(int(axis), send_lo, recv_lo, send_hi, recv_hi, int(nlo), int(nhi))
                return 0
            except Exception as e:  # noqa: BLE001 - reported through the return code
                self.error = e
                self._abort()
                return 1

        def ar(user, op, vals, n):
            try:
                out = self.allreduce(int(op), [vals[i] for i in range(int(n))])
                for i, v in enumerate(out):
                    vals[i] = v
                return 0
            except Exception as e:  # noqa: BLE001
                self.error = e
                self._abort()
                return 1

        self.exchange_fn = abi.EXCHANGE_FN(ex)
        self.allreduce_fn = abi.ALLREDUCE_FN(ar)

    def _abort(self):
        pass


class DistExchange(_Callbacks):
    """This rank's transport over torch.distributed (the process group must be
    initialised).  neighbors: the six ranks of kfvm_block_config.  device: the CUDA
    device of the solver's buffers, or None for host buffers (the CPU restatement
    over gloo)."""

    def __init__(self, neighbors, device=None, group=None):
        super().__init__()
        self.nbr = list(neighbors)
        self.device = device
        self.group = group

    def exchange(self, axis, send_lo, recv_lo, send_hi, recv_hi, nlo, nhi):
        import torch
        import torch.distributed as dist
        d = axis % 3
        lo, hi = self.nbr[2 * d], self.nbr[2 * d + 1]
        if (nlo and lo < 0) or (nhi and hi < 0):
            raise RuntimeError(f"exchange on axis {d} without a neighbour")
        tag = 8 * axis
        ops = []
        if nlo:
            ops.append(dist.P2POp(dist.isend, _view(send_lo, nlo, self.device), lo, self.group, tag + _SIDE_LO))
        if nhi:
            ops.append(dist.P2POp(dist.isend, _view(send_hi, nhi, self.device), hi, self.group, tag + _SIDE_HI))
        if nhi:
            ops.append(dist.P2POp(dist.irecv, _view(recv_hi, nhi, self.device), hi, self.group, tag + _SIDE_LO))
        if nlo:
            ops.append(dist.P2POp(dist.irecv, _view(recv_lo, nlo, self.device), lo, self.group, tag + _SIDE_HI))
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        if self.device is not None:
            # the solver's stream reads the received bytes next
            torch.cuda.current_stream(self.device).synchronize()

    def allreduce(self, op, values):
        import torch
        import torch.distributed as dist
        red = {abi.KFVM_REDUCE_SUM: dist.ReduceOp.SUM, abi.KFVM_REDUCE_MAX: dist.ReduceOp.MAX,
               abi.KFVM_REDUCE_MIN: dist.ReduceOp.MIN}[op]
        t = torch.tensor(values, dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=red, group=self.group)
        return t.cpu().tolist()


class LocalExchange:
    """Blocks of one process, each driven by its own host thread: endpoint(rank,
    neighbors) gives each block its callbacks.  device: the CUDA device of the
    buffers, or None for host buffers.  A block that does not arrive within
    `timeout` seconds breaks the barrier, and every waiting block's step fails."""

    def __init__(self, nranks, device=None, timeout=120.0):
        self.nranks = nranks
        self.device = device
        self.barrier = threading.Barrier(nranks, timeout=timeout)
        self.box = {}
        self.red = [None] * nranks

    def endpoint(self, rank, neighbors):
        return _LocalEndpoint(self, rank, neighbors)


class _LocalEndpoint(_Callbacks):
    def __init__(self, hub, rank, neighbors):
        super().__init__()
        self.hub, self.rank, self.nbr = hub, rank, list(neighbors)

    def _abort(self):
        self.hub.barrier.abort()

    def _sync(self):
        if self.hub.device is not None:
            import torch
            torch.cuda.synchronize(self.hub.device)

    def exchange(self, axis, send_lo, recv_lo, send_hi, recv_hi, nlo, nhi):
        hub, dev, d = self.hub, self.hub.device, axis % 3
        if nlo:
            hub.box[(self.rank, _SIDE_LO)] = _view(send_lo, nlo, dev).clone()
        if nhi:
            hub.box[(self.rank, _SIDE_HI)] = _view(send_hi, nhi, dev).clone()
        self._sync()
        hub.barrier.wait()
        if nlo:
            _view(recv_lo, nlo, dev).copy_(hub.box[(self.nbr[2 * d], _SIDE_HI)])
        if nhi:
            _view(recv_hi, nhi, dev).copy_(hub.box[(self.nbr[2 * d + 1], _SIDE_LO)])
        self._sync()
        hub.barrier.wait()  # nobody refills the mailbox before every block has read it

    def allreduce(self, op, values):
        hub = self.hub
        hub.red[self.rank] = list(values)
        hub.barrier.wait()
        out = list(hub.red[0])
        for r in range(1, hub.nranks):  # in rank order: the same result on every block
            for i, v in enumerate(hub.red[r]):
                if op == abi.KFVM_REDUCE_SUM:
                    out[i] = out[i] + v
                elif op == abi.KFVM_REDUCE_MAX:
                    out[i] = max(out[i], v)
                else:
                    out[i] = min(out[i], v)
        hub.barrier.wait()
        return out


def run_blocks(fns):
    """Run one callable per block in its own thread; re-raise the first failure."""
    errs = [None] * len(fns)

    def body(i):
        try:
            fns[i]()
        except BaseException as e:  # noqa: BLE001
            errs[i] = e

    ts = [threading.Thread(target=body, args=(i,)) for i in range(len(fns))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for e in errs:
        if e is not None:
            raise e
