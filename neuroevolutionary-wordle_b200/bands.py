"""Row bands: one population split by grid rows across ranks, one process per GPU.

The path's dependencies decide the split (the reference runs on one GPU; this follows its data flow):

- evaluation is per individual: a band evaluates its own rows with no communication;
- selection of a child reads the fitness of its Moore neighbourhood (selection_ops.cuh:218-263,
  spatial/grid.hpp:181-218), which crosses band edges: the bands' fitness is all-gathered (4 bytes per
  individual) and every band selects for its own children over the whole grid;
- breeding reads the child's two parents (genome_ops.cuh:386-407), which for a child on a band edge sit up to
  `radius` rows into the neighbouring band: each band receives `halo` rows above and below it from its
  neighbours by point-to-point copies into its own memory (2 * halo * columns genomes per generation).

Children keep their whole-grid indices in every random stream (nwg_band_prepare, nwg_assemble_prepared on a
band), so the bands produce exactly the generation a single runtime holding the whole grid would.

The pure functions here (band layout, halo rows, neighbours) carry the index arithmetic; `exchange_halo` and
`gather_bands` are the two collectives, written against torch.distributed so the same code runs under NCCL on
GPUs and under gloo on the CPU; `BandRuntime` wraps one band's runtime.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import capi


@dataclass(frozen=True)
class BandLayout:
    global_rows: int
    columns: int
    world: int
    rank: int
    halo: int

    @property
    def rows(self) -> int:
        return self.global_rows // self.world

    @property
    def first_row(self) -> int:
        return self.rank * self.rows

    @property
    def cells(self) -> int:
        return self.rows * self.columns

    @property
    def first_cell(self) -> int:
        return self.first_row * self.columns

    @property
    def previous(self) -> int:
        return (self.rank - 1) % self.world

    @property
    def next(self) -> int:
        return (self.rank + 1) % self.world

    def above_rows(self) -> list[int]:
        """Global rows of the halo above the band (the previous band's last rows), top to bottom."""
        return [(self.first_row - self.halo + j) % self.global_rows for j in range(self.halo)]

    def below_rows(self) -> list[int]:
        """Global rows of the halo below the band (the next band's first rows), top to bottom."""
        return [(self.first_row + self.rows + j) % self.global_rows for j in range(self.halo)]

    def parent_rows(self) -> set[int]:
        """Every global row a child of this band may take a parent from: the band and its halo."""
        own = {self.first_row + r for r in range(self.rows)}
        return own | set(self.above_rows()) | set(self.below_rows())


def band_layout(global_rows: int, columns: int, world: int, rank: int, halo: int) -> BandLayout:
    """Equal bands of whole rows. Each band must be at least `halo` rows high (its halo rows then lie in its two
    neighbours only) and the grid must hold the band and both halos as distinct rows."""
    if world < 1 or not 0 <= rank < world or global_rows % world != 0:
        raise ValueError(f"{global_rows} rows do not split into {world} equal bands")
    layout = BandLayout(global_rows, columns, world, rank, halo)
    if halo < 1 or layout.rows < halo or global_rows < layout.rows + 2 * halo:
        raise ValueError(f"bands of {layout.rows} rows cannot carry a halo of {halo} rows in {global_rows} rows")
    return layout


def exchange_halo(layout: BandLayout, first_rows, last_rows, above, below, group=None) -> None:
    """Sends this band's first halo rows to the previous band (its halo below) and its last halo rows to the next
    band (its halo above); receives `above` from the previous band and `below` from the next band.

    Messages between two ranks are matched in the order they are posted, and with two bands the previous and the
    next band are the same rank, so every rank posts: send(last rows -> next), send(first rows -> previous),
    recv(above <- previous), recv(below <- next). Rank k's last rows are then the first message k + 1 receives from
    it (its above halo) and rank k's first rows the second message k - 1 receives from it (its below halo).
    The four operations are posted as one batch (one NCCL group), so no rank blocks on a send its peer has not
    matched yet."""
    import torch.distributed as dist

    ops = [dist.P2POp(dist.isend, last_rows, layout.next, group),
           dist.P2POp(dist.isend, first_rows, layout.previous, group),
           dist.P2POp(dist.irecv, above, layout.previous, group),
           dist.P2POp(dist.irecv, below, layout.next, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def gather_bands(local, out, group=None) -> None:
    """All-gather of equal-sized band arrays into the whole grid's array (band k at offset k * len(local))."""
    import torch.distributed as dist

    dist.all_gather_into_tensor(out, local, group=group)


class _DeviceArray:
    """A device buffer of the runtime seen as a tensor without a copy (the CUDA array interface)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": (count,), "typestr": typestr,
                                         "strides": None, "version": 3}


class BandRuntime:
    """One band of a population split by rows: a runtime holding the band's rows plus room for its halo.

    advance() runs one generation on every rank together: evaluate the band, all-gather fitness, select the band's
    children over the whole grid, exchange halo genomes, breed. `group` is the torch.distributed process group
    (None: the default group)."""

    def __init__(self, layout: BandLayout, action_count: int, stream: int | None = None, group=None):
        import torch

        self.layout = layout
        self.group = group
        self.action_count = action_count
        cells = layout.cells
        halo_cells = layout.halo * layout.columns
        if stream is None:  # the collectives are ordered on torch's current stream: the runtime works on it too
            stream = torch.cuda.current_stream().cuda_stream
        self.rt = capi.Runtime(action_count, cells, layout.columns, stream=stream,
                               slab_slots=2 * cells + 2 * halo_cells)
        self.rt.set_band(layout.global_rows, layout.first_row, layout.halo)
        stride = capi.genome_stride_bytes(action_count)
        self.pitch = (stride + 15) // 16 * 16
        self.population = layout.global_rows * layout.columns
        dev = torch.device("cuda", torch.cuda.current_device())
        self.fitness_all = torch.zeros(self.population, dtype=torch.float32, device=dev)
        self.has_all = torch.zeros(self.population, dtype=torch.uint8, device=dev)
        self.send_first = torch.zeros(halo_cells * self.pitch, dtype=torch.uint8, device=dev)
        self.send_last = torch.zeros_like(self.send_first)
        self.recv_above = torch.zeros_like(self.send_first)
        self.recv_below = torch.zeros_like(self.send_first)
        self.moments = torch.zeros(3, dtype=torch.float64, device=dev)

    def close(self) -> None:
        self.rt.close()

    def bootstrap(self, seed: int, generation_index: int = 0) -> None:
        self.rt.bootstrap(self.layout.cells, seed, generation_index)

    def set_cell_words(self, offsets: np.ndarray, words: np.ndarray) -> None:
        """The whole grid's per-cell word lists (CSR); the band keeps its own cells'."""
        a, b = self.layout.first_cell, self.layout.first_cell + self.layout.cells
        band_offsets = (offsets[a:b + 1] - offsets[a]).astype(np.uint32)
        self.rt.set_cell_words(band_offsets, words[offsets[a]:offsets[b]])

    def local_fitness(self):
        import torch

        f, h, n = self.rt.device_generation()
        return (torch.as_tensor(_DeviceArray(f, n, "<f4"), device="cuda"),
                torch.as_tensor(_DeviceArray(h, n, "|u1"), device="cuda"))

    def gather_fitness(self) -> None:
        fitness, has = self.local_fitness()
        gather_bands(fitness, self.fitness_all, self.group)
        gather_bands(has, self.has_all, self.group)

    def stage_halo(self) -> None:
        """This band's first and last halo rows into the send buffers."""
        h, rows = self.layout.halo, self.layout.rows
        self.rt.band_copy_rows(0, h, self.send_first.data_ptr(), self.pitch)
        self.rt.band_copy_rows(rows - h, h, self.send_last.data_ptr(), self.pitch)

    def install_halo(self) -> None:
        self.rt.band_install_halo(self.recv_above.data_ptr(), self.recv_below.data_ptr(), self.pitch)

    def fitness_moments(self) -> tuple[float, float]:
        """Whole-grid FP64 mean and variance of the last evaluation's fitness, from every band's FP64 moments (one
        all-reduce of three FP64 sums): the statistics the adaptive shard release reads."""
        import torch.distributed as dist

        st = self.rt.stats()
        n = float(self.layout.cells)
        m = st.fitness_mean_fp64
        self.moments.copy_(self.moments.new_tensor([n, n * m, n * (st.fitness_variance_fp64 + m * m)]))
        dist.all_reduce(self.moments, group=self.group)
        total, s, q = (float(v) for v in self.moments.cpu())
        mean = s / total
        return mean, max(q / total - mean * mean, 0.0)

    def advance(self, seed: int, counts, config) -> None:
        """One generation of the whole grid, this band's share (every rank calls it with the same arguments)."""
        self.rt.evaluate(counts)
        self.gather_fitness()
        self.rt.band_prepare(seed, config, self.fitness_all.data_ptr(), self.has_all.data_ptr())
        self.stage_halo()
        exchange_halo(self.layout, self.send_first, self.send_last, self.recv_above, self.recv_below, self.group)
        self.install_halo()
        self.rt.assemble()
