"""The GRAVITY_GPU_B200 blocks of oracle/patch_gravtree.py, on a stand-in of
gravity_tree()'s layout (the statements the script anchors on, in their order;
the test reads nothing of the reference tree).  The patched reference itself is
built by oracle/build_ref.sh and run by tests/test_gizmo_integration.py."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import patch_gravtree  # noqa: E402

STAND_IN = """/* head */
void gravity_tree(void)
{
    int x;
    if(TreeReconstructFlag)
    {
        move_particles(All.Ti_Current);
        rearrange_particle_sequence();
        force_treebuild(NumPart, NULL);
        TreeReconstructFlag = 0;
    }
    setup();
    /* begin main communication and tree-walk loop. comment */
    for(;;) { walk(); }
    myfree(DataNodeList); myfree(DataIndexTable);

    post_processing();
}
"""


def test_blocks_go_where_the_integration_guide_says():
    out = patch_gravtree.patch(STAND_IN)
    # prototypes before the function
    assert out.index("double gravtree_b200_walk(void);") < out.index("void gravity_tree(void)")
    # the build: the device build under the flag, force_treebuild otherwise, after the drift and rearrangement
    b = out.index("        gravtree_b200_build();")
    assert out.index("rearrange_particle_sequence();") < b < out.index("TreeReconstructFlag = 0;")
    assert out.index("#else\n        force_treebuild(NumPart, NULL);\n#endif") > b
    # the walk loop, including its buffer release, is in the #else branch of one device call
    w = out.index("    Costtotal = gravtree_b200_walk();")
    assert out.index("setup();") < w < out.index("/* begin main communication")
    loop_end = out.index("    myfree(DataNodeList); myfree(DataIndexTable);\n#endif\n")
    assert out.index("for(;;) { walk(); }") < loop_end < out.index("post_processing();")
    # the device branch releases the same buffers and skips the per-node cost pass
    dev = out[w:out.index("#else", w)]
    assert "myfree(DataNodeList); myfree(DataIndexTable);" in dev and "TakeLevel = -1;" in dev
    # without the flag the code is unchanged
    plain = "\n".join(l for l in out.splitlines() if "b200" not in l.lower())
    assert "force_treebuild(NumPart, NULL);" in plain and "walk();" in plain


def test_missing_anchor_stops():
    with pytest.raises((SystemExit, ValueError)):
        patch_gravtree.patch(STAND_IN.replace("        force_treebuild(NumPart, NULL);\n", ""))
    with pytest.raises((SystemExit, ValueError)):
        patch_gravtree.patch(STAND_IN.replace("/* begin main communication", "/* loop"))
