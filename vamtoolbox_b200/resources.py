"""vamtoolbox.resources (vamtoolbox/resources.py): the paths of the example images, meshes and saved
toolbox files that ship with the reference toolbox.  This package ships none of those files: a name
resolves inside the folder named by the VAMTOOLBOX_RESOURCES environment variable, or else inside the
``staticresources`` folder of an installed ``vamtoolbox`` package (located without importing it)."""
from __future__ import annotations

import importlib.util
import os
import pathlib
from argparse import ArgumentError

OPTIONS = ["reschart.png", "flower.png", "flower_binarized.png", "trifurcatedvasculature.stl", "bear.stl",
           "thinker.stl", "screwdriver.stl", "ring.stl", "onaxiscylinder.stl", "offaxiscylinder.stl",
           "seq0imagesdir", "sino0.sino", "video0.mp4"]


def _static_dir():
    env = os.environ.get("VAMTOOLBOX_RESOURCES")
    if env:
        return pathlib.Path(env)
    try:
        spec = importlib.util.find_spec("vamtoolbox")
    except (ImportError, ValueError):
        spec = None
    if spec is not None and spec.submodule_search_locations:
        return pathlib.Path(list(spec.submodule_search_locations)[0]) / "staticresources"
    return None


def load(input: str):
    """The path of the named resource (the reference's names, case-insensitive); an unknown name raises
    ArgumentError with the list of names, as in the reference."""
    input = input.lower()
    if input not in OPTIONS:
        raise ArgumentError(None, "Input resource not recognized. Options include: %s" % (OPTIONS,))
    folder = _static_dir()
    if folder is None:
        raise FileNotFoundError("the example resources ship with the reference toolbox: set VAMTOOLBOX_RESOURCES to "
                                "its staticresources folder or install vamtoolbox")
    return str(folder / input)
