"""adapt_boxes (host logic, no GPU): flagged cells below the level cap are
refined, refinement that a flagged finer cell needs is kept, unflagged
refinement goes, the one-cell margins hold (the oracle's topology accepts
every result), and positions next to the domain boundary stay coarse."""
import exahype_b200 as eb
import pyoracle


class _Solver:
    dim = 2


class _Mesh:
    solver = _Solver

    def __init__(self, cells, boxes):
        self.cells, self.boxes = cells, boxes


def test_flagged_cells_are_refined_with_margins():
    m = _Mesh((12, 12), [])
    pos = eb.cell_positions(m)
    assert len(pos) == 144 and pos[1] == (0, (1, 0))
    flags = [p in ((6, 5), (7, 5), (0, 0)) for _, p in pos]  # (0, 0) touches the boundary
    boxes = eb.adapt_boxes(m, flags, 2)
    assert boxes == [(0, (6, 5), (8, 6))]
    m.boxes = boxes
    o = pyoracle.RefinedMesh(2, 3, (12, 12), [1.0, 1.0], level_boxes=boxes)
    assert o.ncells == len(eb.cell_positions(m)) == 144 - 2 + 18


def test_finer_flags_keep_and_grow_refinement_and_unflagged_refinement_goes():
    m = _Mesh((12, 12), [(0, (5, 5), (8, 6))])
    pos = eb.cell_positions(m)
    flags = [lev == 1 and p == (18, 16) for lev, p in pos]
    boxes = eb.adapt_boxes(m, flags, 3)
    assert (1, (18, 16), (19, 17)) in boxes
    level0 = [b for b in boxes if b[0] == 0]
    assert level0 == [(0, (5, 5), (7, 6))]  # (7, 5) coarsened, (5, 5) kept for the margin
    pyoracle.RefinedMesh(2, 3, (12, 12), [1.0, 1.0], level_boxes=boxes)  # a valid topology
    m.boxes = boxes
    assert eb.adapt_boxes(m, [False] * len(eb.cell_positions(m)), 3) == []
