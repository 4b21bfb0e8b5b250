"""Copies a handful of the reference's own test scenes, with the meshes and textures they
load, into tests/golden/refscenes/ for the GPU parity tests of the scene reader.

    python tests/golden/make_reference_scenes.py REFERENCE_ROOT

The scenes come from the reference's testing/scenes/ directory unchanged (they are its
render-regression inputs); together they exercise COLLADA meshes (unitcube.dae,
cornelbox.dae), OBJ meshes with texture coordinates, a diffuse PNG texture, parallel and
uniform area emitters, analytic spheres and nested homogeneous media.  The tests read only
the copies, never the reference tree.
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SCENES = ["nested_media1.nff", "cornelbox_translucentsphere.nff", "refractive_sphere_caustics.nff",
          "refract_beam_at_cube.nff", "cubelight.nff", "litcorner2.nff", "medium_in_medium.nff"]
ASSETS = ["unitcube.dae", "cornelbox.dae", "unitrectangle.obj", "checkerboard_bright_256.png"]


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    src = Path(argv[1]) / "testing" / "scenes"
    dst = HERE / "refscenes"
    dst.mkdir(exist_ok=True)
    for name in SCENES + ASSETS:
        shutil.copyfile(src / name, dst / name)
    print(f"copied {len(SCENES)} scenes and {len(ASSETS)} assets to {dst}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
