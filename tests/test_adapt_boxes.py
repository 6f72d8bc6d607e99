"""adapt_boxes (host logic, no GPU), with the reference's refinement
controls: cells that answer REFINE below the level cap are refined, KEEP
leaves the refinement as it is, a refined position goes only when all of its
children answer ERASE (a refined child vetoes too), the one-cell margins hold
(the oracle's topology accepts every result), and positions next to the
domain boundary stay coarse."""
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


def test_finer_refine_grows_refinement_and_keep_keeps_it():
    m = _Mesh((12, 12), [(0, (5, 5), (8, 6))])
    pos = eb.cell_positions(m)
    controls = [eb.REFINE if (lev == 1 and p == (18, 16)) else eb.KEEP for lev, p in pos]
    boxes = eb.adapt_boxes(m, controls, 3)
    assert (1, (18, 16), (19, 17)) in boxes
    assert [b for b in boxes if b[0] == 0] == [(0, (5, 5), (8, 6))]  # KEEP everywhere else: nothing coarsens
    pyoracle.RefinedMesh(2, 3, (12, 12), [1.0, 1.0], level_boxes=boxes)  # a valid topology
    m.boxes = boxes
    # KEEP from every cell (and booleans False) leaves the refinement as it is
    n = len(eb.cell_positions(m))
    assert eb.adapt_boxes(m, [eb.KEEP] * n, 3) == boxes
    assert eb.adapt_boxes(m, [False] * n, 3) == boxes


def test_erase_needs_every_child_and_refined_children_veto():
    m = _Mesh((12, 12), [(0, (5, 5), (8, 6))])
    pos = eb.cell_positions(m)
    kids_of_75 = {(x, y) for x in range(21, 24) for y in range(15, 18)}
    # every child of (7, 5) erases; (6, 5) has one child that keeps; (5, 5) all erase but one refines
    controls = []
    for lev, p in pos:
        if lev == 1 and p in kids_of_75:
            controls.append(eb.ERASE)
        elif lev == 1 and p == (18, 16):
            controls.append(eb.KEEP)
        elif lev == 1 and p == (15, 15):
            controls.append(eb.REFINE)
        elif lev == 1:
            controls.append(eb.ERASE)
        else:
            controls.append(eb.KEEP)
    boxes = eb.adapt_boxes(m, controls, 3)
    level0 = [b for b in boxes if b[0] == 0]
    # (7, 5) goes; (6, 5) stays (a KEEP child vetoes); (5, 5) stays (a REFINE child)
    # and so do the parents its new level-1 refinement needs for its margin
    assert (0, (7, 5), (8, 6)) not in level0 and all(not (b[1][0] <= 7 < b[2][0] and b[1][1] <= 5 < b[2][1])
                                                      for b in level0)
    assert any(b[1][0] <= 6 < b[2][0] and b[1][1] <= 5 < b[2][1] for b in level0)
    assert (1, (15, 15), (16, 16)) in boxes
    pyoracle.RefinedMesh(2, 3, (12, 12), [1.0, 1.0], level_boxes=boxes)
    # all leaves erase: the refined level-1 position (15, 15) goes, but it still
    # vetoes the erase of its parent (5, 5) in this pass (one level per pass,
    # as the reference's children vote only on their direct parent)
    m.boxes = boxes
    assert eb.adapt_boxes(m, [eb.ERASE] * len(eb.cell_positions(m)), 3) == [(0, (5, 5), (6, 6))]
    # everything erases on a mesh refined one level deep: no refinement left
    m1 = _Mesh((12, 12), [(0, (5, 5), (8, 6))])
    assert eb.adapt_boxes(m1, [eb.ERASE] * len(eb.cell_positions(m1)), 3) == []
