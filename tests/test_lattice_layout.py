"""The lattice form's layout and work split, checked on the CPU.

The lattice march (nh-flood-2d_b200/csrc/nhf_lattice.cu) splits a uniform
grid into strips of 28 owned columns (a warp's lanes 2..29, lanes 0, 1, 30,
31 being halo) and chunks of ``rows`` rows, and gives the CFL sides on strip
and chunk edges to the close pass. Bit-exact results need every lattice
point (cell and its west/south sides) written by exactly one warp, every
interior side's CFL candidate taken exactly once, and every load inside
the allocated lattice. This restates the planner's formulas and the
kernels' index ranges and checks those three properties over grid shapes
and chunk heights, including the ones the GPU tests force through the
planner's knobs:

  layout      nhf_lattice.cu:720-725 (strips, lx = 28 strips + 4,
              ly = chunks x rows + 5, cell (i, j) at (j + 2) lx + i + 2)
  march       nhf_lattice.cu:303-380 (own lanes, rows y0 - 3 .. y1 - 1,
              loads of rows y + 1 .. y + 3, CFL of west sides at lanes > 2
              and of south sides at rows > y0, edge records)
  close       nhf_lattice.cu:480-495 (west sides of each strip's first
              column from the edge records, south sides of each chunk's
              first row)
"""
import numpy as np
import pytest

K_OUT, K_LANES, K_WEST = 28, 32, 2


def layout(nx, ny, rows):
    strips = (nx + 1 + K_OUT - 1) // K_OUT
    chunks = (ny + 1 + rows - 1) // rows
    return strips, chunks, strips * K_OUT + K_WEST + 2, chunks * rows + 5


def march(nx, ny, rows):
    """Per lattice point: how often it is written, how often its west and
    south sides' CFL candidates are taken; the extreme rows and columns any
    load touches."""
    strips, chunks, lx, ly = layout(nx, ny, rows)
    written = np.zeros((ly, lx), np.int32)
    cfl_w = np.zeros((ly, lx), np.int32)
    cfl_s = np.zeros((ly, lx), np.int32)
    edge = np.zeros((strips, chunks * rows), np.int32)
    lo_row, hi_row = ly, -1
    hi_col = (strips - 1) * K_OUT + K_LANES - 1
    for c in range(chunks):
        y0 = 2 + c * rows
        y1 = y0 + rows
        lo_row = min(lo_row, y0 - 2)  # the prologue loads rows y0 - 2 and y0 - 1
        for y in range(y0 - 3, y1):
            hi_row = max(hi_row, y + 3)  # iteration y loads row y + 3 for the next one
            if y < y0:
                continue
            for s in range(strips):
                x0 = s * K_OUT
                written[y, x0 + 2:x0 + 2 + K_OUT] += 1
                cfl_w[y, x0 + 3:x0 + 2 + K_OUT] += 1          # lane > 2
                if y > y0:
                    cfl_s[y, x0 + 2:x0 + 2 + K_OUT] += 1      # row > y0
                edge[s, y - 2] += 1
    # the close pass: strip edges from the records (strip 0's west is the border),
    # chunk edges from the lattice
    for s in range(1, strips):
        cfl_w[2:2 + chunks * rows, s * K_OUT + 2] += 1
    for c in range(chunks):
        cfl_s[2 + c * rows, 2:2 + strips * K_OUT] += 1
    return dict(written=written, cfl_w=cfl_w, cfl_s=cfl_s, edge=edge, lo_row=lo_row, hi_row=hi_row,
                hi_col=hi_col, lx=lx, ly=ly)


SHAPES = [(90, 90, 4), (90, 90, 7), (90, 90, 16), (48, 48, 4), (64, 64, 16), (33, 1030, 16), (1030, 33, 8),
          (256, 256, 4), (1024, 1024, 16), (2048, 2048, 16), (300, 17, 256)]


@pytest.mark.parametrize('nx,ny,rows', SHAPES)
def test_every_point_and_side_once_and_loads_in_bounds(nx, ny, rows):
    r = march(nx, ny, rows)
    lx, ly = r['lx'], r['ly']
    # cells at rows 2..ny+1, columns 2..nx+1; the points one beyond carry the
    # east and north boundary sides
    cells = (slice(2, ny + 3), slice(K_WEST, nx + K_WEST + 1))
    assert (r['written'][cells] == 1).all()
    assert r['written'].max() == 1
    # every west side of columns 3..nx+1 and south side of rows 3..ny+1, the
    # sides between two cells (the only ones a CFL candidate can come from),
    # exactly once
    assert (r['cfl_w'][2:ny + 2, K_WEST + 1:nx + K_WEST + 1] == 1).all()
    assert (r['cfl_s'][3:ny + 2, K_WEST:nx + K_WEST] == 1).all()
    assert r['cfl_w'].max() == 1 and r['cfl_s'].max() == 1
    # loads stay inside the allocated lattice
    assert r['lo_row'] >= 0 and r['hi_row'] <= ly - 1
    assert r['hi_col'] <= lx - 1
    # every edge record is written once per step, so none is stale
    assert (r['edge'] == 1).all()
    # the planner's 2^30 bound keeps 32-bit lattice indices exact
    assert lx * ly < 2 ** 31


def test_lane_counters_fit_their_fields():
    """A lane packs its limited-cell, limited-face and wet-cell counts into
    one 32-bit word (bits 0-9, 10-19, 20-31; nhf_lattice.cu:288-290). Per
    chunk a lane counts at most one limited cell, two limited faces (its
    west and south sides) and one wet cell per row, and the planner caps
    the rows at 256 (nhf_lattice.cu:667)."""
    max_rows = 256
    assert max_rows < 2 ** 10 and 2 * max_rows < 2 ** 10 and max_rows < 2 ** 12
