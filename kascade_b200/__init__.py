"""kascade_b200: list ranking and tree rooting on one NVIDIA B200 (sm_100a).

A from-scratch GPU implementation of the list-ranking / tree-rooting hot path
of niklas-uhl/kascade.  The compute path is libkascade_b200.so (hand-written
CUDA behind a C ABI, include/kascade_b200.h); this package is the Python
mirror of the reference's lib/kascade functions over that ABI.
"""
from ._lib import LIB_PATH, KascadeError, declared_symbols, lib  # noqa: F401
from .api import (  # noqa: F401
    FOREST_CATERPILLAR,
    FOREST_RRT,
    LAYOUT_IDENTITY,
    LAYOUT_RANDOM,
    LAYOUT_RUNS,
    SEG_FOREST,
    SEG_LIST,
    Algorithm,
    B200Ranking,
    BatchPlan,
    Context,
    EulerTourConfig,
    GpuTuning,
    PointerDoublingConfig,
    RulerSelectionStrategy,
    Server,
    SparseRulingSetConfig,
    async_pointer_doubling,
    batch_sizes,
    gen_batch,
    get_class_launch,
    get_size_classes,
    load_tuning,
    set_class_launch,
    make_segments,
    rank_batch,
    set_size_classes,
    STATS_BASIC,
    STATS_EXTENSIVE,
    STATS_NONE,
    STATS_REDUCED_EXTENSIVE,
    compute_euler_tour,
    compute_stats,
    default_context,
    gen_forest,
    gen_list,
    gen_weights,
    is_list,
    local_pointer_chasing,
    pack,
    pointer_doubling,
    rank_list,
    rank_list_host,
    rank_on_root,
    rank_via_euler_tour,
    rma_pointer_doubling,
    root_forest,
    root_forest_host,
    set_initial_ranking_state,
    sparse_ruling_set,
    unpack,
)

__version__ = "0.1.0"
