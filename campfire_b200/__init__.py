"""campfire_b200: the campfire gas step (BoccheseGiacomo/campfire, js/fluid.js +
shaders/*.wgsl) as hand-written sm_100a CUDA kernels behind a C ABI
(include/campfire_gas.h, libcampfire_gas.so), with a Python mirror of the
reference's FluidSim interface."""
from ._lib import (CampfireError, SOLVE_FIXED, SOLVE_FP64, SOLVE_TOL, declared_symbols, device_count, lib)
from .fluid import (SCENE_WIDTH, STAGES, TILE_SHAPES, Batch, FluidSim, Server, autotune, autotune_tiles, field_hash,
                    generate_scene, load_scene)
from .render import GROUND, VIEWS, Renderer, write_png

__all__ = ["CampfireError", "FluidSim", "Batch", "Server", "autotune", "autotune_tiles", "TILE_SHAPES", "field_hash", "generate_scene", "load_scene", "lib", "device_count",
           "declared_symbols", "Renderer", "VIEWS", "GROUND", "write_png", "SOLVE_FIXED", "SOLVE_TOL", "SOLVE_FP64", "SCENE_WIDTH", "STAGES"]
