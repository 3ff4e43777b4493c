#!/usr/bin/env python3
"""Write GIZMO's gravity/gravtree.c with the GRAVITY_GPU_B200 blocks added.

TEST INFRASTRUCTURE ONLY (run by build_ref.sh): it reads the reference's own
gravity/gravtree.c from the source tree's mirror, adds the compile-flag
blocks that INTEGRATION.md documents, and writes the result over the mirror's
symlink in the temporary build directory (never into this repository).  With
-DGRAVITY_GPU_B200 the reference's own gravity_tree() then calls the B200
library through gizmo-public_b200/host/gravtree_b200.c and keeps all of its
own post-processing (x G, OldAcc, the switch to the relative criterion, the
2LPT guard, timing logs; gravtree.c:475-654), its particle drift and
rearrangement before a rebuild (move_particles, rearrange_particle_sequence;
gravtree.c:71-72) and its buffer handling.

The blocks, anchored on statements of gravity_tree() (gravtree.c:51-654):
  1. prototypes of the two host functions, before gravity_tree();
  2. the tree construction force_treebuild(NumPart, NULL) (gravtree.c:74)
     becomes gravtree_b200_build();
  3. the walk / export loop, from the comment that opens it to the release of
     its buffers (gravtree.c:137-457), becomes one call of
     gravtree_b200_walk(), which fills P[].GravAccel and P[].Potential
     (pre-G) for the active particles and returns the interaction count; the
     buffers are released the same way, and the per-node cost bookkeeping that
     reads the CPU tree (gravtree.c:460-470) is skipped (TakeLevel = -1: the
     device walk keeps no per-node costs).
Every anchor must occur exactly where expected, or the script stops.
"""
import os
import sys

PROTO = """#ifdef GRAVITY_GPU_B200
void gravtree_b200_build(void);
double gravtree_b200_walk(void);
#endif
"""

BUILD_OLD = "        force_treebuild(NumPart, NULL);\n"
BUILD_NEW = """#ifdef GRAVITY_GPU_B200
        gravtree_b200_build();   /* keys, sort, oct-tree and FP64 moments on the GPU */
#else
        force_treebuild(NumPart, NULL);
#endif
"""

LOOP_START = "    /* begin main communication and tree-walk loop."
LOOP_END = "    myfree(DataNodeList); myfree(DataIndexTable);\n"
WALK_NEW = """#ifdef GRAVITY_GPU_B200
    Costtotal = gravtree_b200_walk();   /* every active particle: pre-G GravAccel and Potential in P[] */
    myfree(DataNodeList); myfree(DataIndexTable);
    TakeLevel = -1;   /* the device walk keeps no per-node costs */
#else
"""


def patch(src):
    fn = src.index("void gravity_tree(void)\n{")
    tree_if = src.index("    if(TreeReconstructFlag)\n", fn)
    b = src.index(BUILD_OLD, tree_if)
    if b > src.index("TreeReconstructFlag = 0;", tree_if):
        raise SystemExit("patch_gravtree: force_treebuild is not inside the rebuild block")
    ls = src.index(LOOP_START, b)
    le = src.index(LOOP_END, ls) + len(LOOP_END)
    if src.count(LOOP_START) != 1 or src.count(BUILD_OLD) != 1:
        raise SystemExit("patch_gravtree: anchors not unique")
    out = (src[:fn] + PROTO + "\n" + src[fn:b] + BUILD_NEW + src[b + len(BUILD_OLD):ls] + WALK_NEW +
           src[ls:le] + "#endif\n" + src[le:])
    return out


def main():
    if len(sys.argv) != 3:
        raise SystemExit("usage: patch_gravtree.py <reference gravtree.c> <output>")
    src = open(sys.argv[1]).read()
    out = patch(src)
    # the output path may be a symlink into the reference tree: replace the
    # link, never write through it
    if os.path.islink(sys.argv[2]):
        os.unlink(sys.argv[2])
    with open(sys.argv[2], "w") as f:
        f.write(out)


if __name__ == "__main__":
    main()
