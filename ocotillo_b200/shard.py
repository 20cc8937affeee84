"""Multi-GPU sharding of a block's columns (one process per GPU).

The (column, wavelength) items are independent, so a block is split into contiguous column
ranges, one per rank, as the reference splits its domain into procx x procy blocks
(source/flux_feautrier.f90:132-133); there is no exchange during the solve.  The only
collective is the optional gather of the emergent-flux planes at the end.
"""
import numpy as np


def column_range(ncol, rank, world):
    """Contiguous, balanced range [c0, c1) of the ncol columns owned by `rank`."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(ncol, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def local_columns(rho, T, rank, world):
    """The rank's columns of (nx, ny, nz) inputs as (1, n_local, nz) blocks (column order
    col = ix*ny + iy, as the reference's loops), with the range."""
    nx, ny, nz = rho.shape
    c0, c1 = column_range(nx * ny, rank, world)
    r = rho.reshape(nx * ny, nz)[c0:c1].reshape(1, c1 - c0, nz)
    t = T.reshape(nx * ny, nz)[c0:c1].reshape(1, c1 - c0, nz)
    return r, t, (c0, c1)


def gather_planes(local, ncol, world, group=None):
    """All-gathers per-rank emergent-flux planes (nw, n_local) into (nw, ncol) on every rank
    (torch tensors; uneven ranges are padded to the largest)."""
    import torch
    import torch.distributed as dist
    nw = local.shape[0]
    sizes = [column_range(ncol, r, world) for r in range(world)]
    width = max(c1 - c0 for c0, c1 in sizes)
    pad = torch.zeros((nw, width), dtype=local.dtype, device=local.device)
    pad[:, :local.shape[1]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:, :c1 - c0] for p, (c0, c1) in zip(parts, sizes)], dim=1)


def solve_sharded(solve, rho, T, rank, world, group=None):
    """Solves the rank's columns with `solve(rho_local, T_local) -> {'Vtop', 'Vbot'}` (arrays of
    shape (nw, 1, n_local)) and returns the full emergent-flux planes (nw, nx, ny) on every
    rank as numpy arrays."""
    import torch
    nx, ny, _ = rho.shape
    if nx * ny < world:  # every rank sees the same shapes, so all refuse before any collective
        raise ValueError(f"{nx * ny} columns cannot give each of {world} ranks one")
    r, t, _ = local_columns(rho, T, rank, world)
    out = solve(r, t)
    res = {}
    for k in ("Vtop", "Vbot"):
        loc = torch.as_tensor(np.ascontiguousarray(out[k]).reshape(out[k].shape[0], -1))
        res[k] = gather_planes(loc, nx * ny, world, group).numpy().reshape(-1, nx, ny)
    return res
