"""Multi-rank host logic: one process per GPU.

Three pieces of the reference's MPI parallelisation are mirrored:
  - the (spin, k, band) targets of an apply are split over ranks by k-point,
    round robin, through the ownership mask of tcg_apply
    (Parallelization::set_orbital_parallelization, parallelization.cpp:127-172);
  - the occupied-pair stage of tc3a2a4b2b5 is split over the occupied sources
    (q1, i1), and each rank's partial intermediate grids are summed over ranks
    before the rotation / local-potential half runs on every rank
    (calc_hamiltonian_tc3a2a4b2b5.cpp:214-235 split, :490-493 and :649-659
    MPI_Allreduce).  The sum is one torch.distributed all_reduce (NCCL on the
    GPU) of the library's device buffer;
  - the reduction of H phi over ranks that closes calc_hamiltonian::all
    (MPI_Reduce to rank 0, calc_hamiltonian_all.cpp:164-197): each rank's
    packed H1 / H2 / H3 holds its own bands (zero elsewhere), and
    reduce_h sums them with one collective per array, on the device.
"""
import numpy as np


def owned_mask(system, world, rank):
    """tcg_apply ownership flags: band-applies of k-point k belong to rank k % world."""
    flags = []
    for s in range(system.nspin):
        for k in range(system.nk_irr):
            flags += [1 if (k % world) == rank else 0] * int(system.nb_apply[s][k])
    return np.array(flags, dtype=np.uint8)


class _DeviceBuffer:
    """Zero-copy view of a device buffer of float64 for torch.as_tensor."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes // 8,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(ptr, nbytes, device):
    import torch
    return torch.as_tensor(_DeviceBuffer(ptr, nbytes), device=device)


def sharded_qp_stage(ctx, group=None, view=None):
    """Compute the tc3a2a4b2b5 occupied-pair stage split over the ranks of
    `group` (torch.distributed): this rank's share, an in-place all_reduce
    (sum) of the partial grids, then the second half on every rank.
    view(ptr, nbytes) -> tensor over the device buffer (default: a CUDA view
    on the current device)."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    ptr, nbytes = ctx.qp_partial(rank, world)
    if view is None:
        buf = device_view(ptr, nbytes, torch.device("cuda", torch.cuda.current_device()))
    else:
        buf = view(ptr, nbytes)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    if buf.is_cuda:
        torch.cuda.synchronize(buf.device)
    ctx.qp_finish()


def reduce_h(arrays, group=None, dst=None):
    """Sum the ranks' packed H phi arrays (torch tensors, complex128 or their
    float64 views; on the GPU for NCCL) in place: all ranks receive the sum
    (dst None) or only rank dst (the reference's MPI_Reduce to rank 0)."""
    import torch
    import torch.distributed as dist
    for a in arrays:
        if a is None:
            continue
        buf = torch.view_as_real(a) if a.is_complex() else a
        if dst is None:
            dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        else:
            dist.reduce(buf, dst=dst, op=dist.ReduceOp.SUM, group=group)
