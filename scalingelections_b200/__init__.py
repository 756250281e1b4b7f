"""Schulze-method hot path (ballot tally, widest-path closure, ranking) on B200 (sm_100a).

A from-scratch CUDA implementation behind the entry points that ashvardanian/ScalingElections'
``scaling_elections.py`` uses. ``scalingelections_b200.dropin`` holds a ``scaling_elections``
module with the reference's native-module surface.
"""
from .api import (  # noqa: F401
    Ballots,
    ClosureStream,
    LANES_AUTO,
    LANES_U16,
    LANES_U32,
    SchulzeError,
    SchulzeResult,
    build_pairwise_preferences,
    closure_workspace_bytes,
    compute_strongest_paths,
    get_winner_and_ranking,
    log_gpus,
    rank_device,
    schulze,
    strongest_paths_device,
    tally_device,
    tally_workspace_bytes,
)

__version__ = "0.1.0"
