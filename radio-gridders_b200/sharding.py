"""Splitting one imaging job over several GPUs (one process per GPU,
torch.distributed for the collectives).  The reference images on one GPU;
these are the partitions its work units allow:

* W-towers: towers are independent until the add-back, so each rank grids a
  load-balanced share of the towers (rg_wtowers_partition over
  rg_wtowers_tower_loads) into its own FP64 master grid and one reduce sums
  them (`tower_parts`, `reduce_grid`).
* W-projection: gridding is linear in the visibilities, so each rank grids a
  contiguous share of them (`vis_share`) and the same reduce sums the grids.
* Direct DFT: every pixel is independent, so each rank computes a band of
  image rows (`dft_row_ranges`, rg_dft_image_rows) and the bands are gathered
  (`gather_rows`).

Every rank calls the same collectives in the same order.  Grids are complex128
torch tensors (they travel as their real view); bands are float64 tensors.
"""
import importlib


def tower_parts(vis_per_tower, floors_per_tower, world):
    """Part (rank) of each tower: the library's deterministic balance of
    visibilities and active w-floors, the same on every rank."""
    rg = importlib.import_module("radio-gridders_b200")
    return rg.partition_towers(vis_per_tower, floors_per_tower, world)


def vis_share(nvis, world, rank):
    """[begin, end) of rank's contiguous share of nvis visibilities (sizes
    differ by at most one)."""
    base, extra = divmod(int(nvis), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def dft_row_ranges(grid_size, world, align=32):
    """[(row0, nrows)] per rank: contiguous bands of image rows, each starting
    on a multiple of `align` (the DFT's tile height, so each band's pixels
    equal the whole image's bit for bit), as even as that allows."""
    tiles = -(-int(grid_size) // align)
    out = []
    for r in range(world):
        t0 = r * tiles // world
        t1 = (r + 1) * tiles // world
        row0 = min(t0 * align, grid_size)
        out.append((row0, min(t1 * align, grid_size) - row0))
    return out


def reduce_grid(grid, world, dst=0):
    """Sum the ranks' FP64 master grids onto rank dst (one collective)."""
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.reduce(torch.view_as_real(grid), dst=dst)


def gather_rows(band, grid_size, ranges, world):
    """All ranks' row bands (band: this rank's nrows x grid_size float64
    tensor) into the full image on every rank (one all-gather of bands padded
    to the largest)."""
    import torch
    if world == 1:
        return band
    import torch.distributed as dist
    most = max(n for _, n in ranges)
    pad = torch.zeros((most, grid_size), dtype=band.dtype, device=band.device)
    pad[: band.shape[0]] = band
    out = torch.empty((world * most, grid_size), dtype=band.dtype, device=band.device)
    dist.all_gather_into_tensor(out, pad)
    image = torch.empty((grid_size, grid_size), dtype=band.dtype, device=band.device)
    for r, (row0, n) in enumerate(ranges):
        image[row0:row0 + n] = out[r * most:r * most + n]
    return image


__all__ = ["tower_parts", "vis_share", "dft_row_ranges", "reduce_grid", "gather_rows"]
