"""B200-native implementation of steel-webgpu's ``Sim.step`` hot path."""
from .builder import SceneBuilder, convex_hull, load_scene, LoadedScene  # noqa: F401
from .packer import pack, Packed  # noqa: F401
