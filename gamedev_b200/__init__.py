"""gamedev_b200: B200-native swarm collision path (index build, exact top-K, pair rates,
frozen-bath event chain) behind a C ABI (include/gd_b200.h, libgd_b200.so)."""

from ._lib import (GD_KERNEL_CONSTANT, GD_KERNEL_CUSTOM, GD_KERNEL_LINEAR, GD_KERNEL_PRODUCT,
                   GD_SEARCH_KDTREE, GD_SEARCH_MORTON, GdConfig, GdError, default_config, load)
from .swarm import (PARTICLE_DTYPE, STATIC_MAX_PARTICLES, RadiusModel, SwarmBatch, SwarmCollision, frame_name,
                    knn_static, load_checkpoint, particles_from_file_layout, particles_to_device,
                    particles_to_file_layout, rng_state_bytes, rng_uniforms, rngstate_init, save_checkpoint,
                    save_variables, wedge_info)

__all__ = [
    "GdConfig", "GdError", "SwarmCollision", "SwarmBatch", "RadiusModel", "default_config", "load", "rngstate_init",
    "rng_state_bytes", "rng_uniforms", "particles_to_device", "PARTICLE_DTYPE", "knn_static",
    "STATIC_MAX_PARTICLES", "frame_name", "particles_to_file_layout", "particles_from_file_layout",
    "save_checkpoint", "load_checkpoint", "wedge_info", "save_variables",
    "GD_SEARCH_KDTREE", "GD_SEARCH_MORTON",
    "GD_KERNEL_CONSTANT", "GD_KERNEL_LINEAR", "GD_KERNEL_PRODUCT", "GD_KERNEL_CUSTOM",
]
