"""Command-line simplification of an OBJ or PLY mesh, with the options of the
reference's example.py:13-21:

    python -m pamo_b200.cli -i in.obj -o out.obj -r 0.1 [-mv 0] [--disable_stage1] [--disable_stage3]
"""
from __future__ import annotations

import argparse
import sys
import time


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m pamo_b200.cli")
    ap.add_argument("-i", "--input", type=str, required=True)
    ap.add_argument("-o", "--output", type=str, required=True)
    ap.add_argument("-r", "--ratio", type=float, default=0.1)
    ap.add_argument("-mv", "--min-vertex", type=int, default=0)
    ap.add_argument("--disable_stage1", action="store_true", help="Disable remeshing")
    ap.add_argument("--disable_stage3", action="store_true", help="Disable safe projection")
    args = ap.parse_args(argv)

    import torch

    from . import PaMO
    from .meshio import load_mesh, save_mesh

    mesh = load_mesh(args.input)
    print(f"# of input verts : {len(mesh.vertices)}")
    print(f"# of input faces : {len(mesh.faces)}")
    pamo = PaMO(mesh, use_stage1=not args.disable_stage1, use_stage3=not args.disable_stage3)
    start = time.time()
    verts, faces = pamo.run(torch.from_numpy(mesh.vertices).float().cuda(), torch.from_numpy(mesh.faces).int().cuda(),
                            min_verts=args.min_vertex, ratio=args.ratio)
    print("Total time: ", time.time() - start)
    print(f"# of output verts : {len(verts)}")
    print(f"# of output faces : {len(faces)}")
    save_mesh(args.output, verts, faces)
    return 0


if __name__ == "__main__":
    sys.exit(main())
