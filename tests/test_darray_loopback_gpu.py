"""The CUDA pack / unpack / local-copy kernels of a multi-rank
redistribution, on one GPU: this rank's workspace of a world-size 2 or 3
blocking, its pack plan against the send buffers the oracle's pack_data
builds (byte-exact, x fastest, per-peer offsets in walk order), and, with
the receive buffer loaded with what the oracle's peers would send (the
exchange replaced by a loopback), its local-copy and unpack plans against
the array itself.  Reference: pack_kernel! / unpack_kernel! /
gpu_pack_peer! / gpu_unpack_peer! (src/fftgpu.jl:417-480), pack_data! /
unpack_data! (src/fft.jl:180-214)."""
import numpy as np
import pytest
import torch

import dfft
import dfft_oracle as oracle
from dfft.darray import CudaCopier
from helpers import rand, to_gpu

pytestmark = pytest.mark.gpu

CASES = [
    (2, 0, (8, 6, 4), (8, 6, 1), (2, 6, 4)),        # slab -> slab
    (2, 1, (8, 8, 8), (8, 4, 4), (4, 8, 4)),        # pencil x -> pencil y
    (3, 1, (10, 9, 7), (10, 3, 2), (3, 9, 3)),      # ragged blocks
    (3, 2, (64, 48, 40), (64, 48, 8), (16, 48, 40)),
    (2, 0, (33, 17, 12), (33, 5, 4), (7, 17, 5)),
]


def _mailbox(A, shape, bsrc, bdst, world):
    """(sender, receiver) -> the flat buffer the oracle's ranks exchange."""
    src = oracle.distribute(A, oracle.blocks(shape, bsrc, world))
    dst = oracle.blocks(shape, bdst, world)
    box = {}
    for r in range(world):
        ws = oracle.create_workspace(src, dst, r)
        for peer, pats in ws.send_peers.items():
            buf = np.empty(ws.send_sizes[peer], dtype=A.dtype)
            for p in pats:
                oracle.pack_data(buf, src.chunks[p.src_idx], p.src_indices, p.buffer_offset)
            box[(r, peer)] = buf
    return box


@pytest.mark.parametrize("world,rank,shape,bsrc,bdst", CASES)
def test_pack_and_unpack_kernels(world, rank, shape, bsrc, bdst):
    A = rand(shape, np.complex64, seed=sum(shape) + rank)
    box = _mailbox(A, shape, bsrc, bdst, world)
    g = to_gpu(A)
    DA = dfft.distribute(g, dfft.Blocks(*bsrc), rank=rank, world=world)
    DB = dfft.empty_darray(shape, dfft.Blocks(*bdst), g.dtype, rank=rank, world=world)
    ws = dfft.create_gpu_workspace(DA, DB)
    cop = CudaCopier()
    # pack: every send to every peer, sorted by rank, one launch
    want_send = [box[(rank, p)] for p in ws.send_ranks]
    if want_send:
        cop.run(ws, "pack", DA, DB)
        torch.cuda.synchronize()
        got = ws.send_buffer.cpu().numpy()
        assert np.array_equal(got, np.concatenate(want_send))
    # loopback exchange: the receive buffer gets what the peers send this rank
    want_recv = [box[(p, rank)] for p in ws.recv_ranks]
    if want_recv:
        ws.recv_buffer.copy_(torch.from_numpy(np.concatenate(want_recv)))
    cop.run(ws, "local", DA, DB)
    if want_recv:
        cop.run(ws, "unpack", DA, DB)
    torch.cuda.synchronize()
    for i in DB.local_indices:
        d = DB.subdomains[i]
        exp = A[d[0].start:d[0].stop, d[1].start:d[1].stop, d[2].start:d[2].stop]
        assert np.array_equal(DB.chunks[i].cpu().numpy(), exp), i
