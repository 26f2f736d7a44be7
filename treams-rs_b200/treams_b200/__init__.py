"""Python host API over the B200 C-ABI library ``libtreams_b200.so``.

Mirrors the treams-rs entry points of the cluster hot path (python/treams_rs and the
``_native`` bindings): dense sphere-cluster factors with repeated solves
(``sphere_cluster_factor``), the matrix-free cluster (``SphereCluster``), translation
blocks (``sw.translate_block``), plane-wave incidence, cross sections, and the 2D Ewald
lattice sums (``lattice.lsumsw2d``). Every call runs on the GPU; there is no CPU path,
and importing fails loudly when the library has not been built.
"""
from ._lib import (  # noqa: F401
    FP64,
    MIXED,
    Certificate,
    Context,
    InteractionFactor,
    SphereCluster,
    TreamsCudaError,
    batch_solve,
    cluster_apply,
    cluster_operator,
    cross_sections,
    default_context,
    LearnedProblem,
    learned_weight_count,
    library_path,
    mie_blocks,
    plane_wave_expansion,
    sphere_cluster_factor,
    translation_block,
)
from . import lattice, sw  # noqa: F401,E402
