"""The reference's one published result, reproduced: the standalone octree
build of a float32 Plummer sphere with N = 20,000,000 and NLEAF = 16 has
596,463 nodes, 4,041,848 leaves, 4,638,311 cells and 15 levels
(treebuild/readme:33-39, plummer.h's default seed).  The tree shape depends
on every particle's octant path, so equality pins the input generator and the
octree build against the reference's own output at full size."""
import pytest

pytestmark = pytest.mark.gpu


def test_tree_shape_matches_the_published_build():
    import bonsai2_b200 as B
    n = 20_000_000
    p, v = B.plummer(n, 19810614)
    t = B.Treecode(eps=0.01, theta=0.5, nleaf=16)
    t.alloc(n)
    t.h_ptclPos[:] = p
    t.h_ptclVel[:] = v
    t.ptcl_h2d()
    t.buildTree(16)
    info = t.tree_info()
    assert (info["nnodes"], info["nleaves"], info["ncells"], info["nlevels"]) == (596463, 4041848, 4638311, 15)
    assert t.synchronize() == 0
    t.close()
