"""Drop-in ``scaling_elections`` module: the native-module surface that the reference's
``scaling_elections.py`` imports (scaling_elections.cu:991-1039, imported at py:30-31),
served by the sm_100a kernels of ``scalingelections_b200``.

Put the directory holding this package first on ``sys.path`` (or place the package next to
the reference's script: a package directory wins over a same-named ``.py`` module in the same
directory). ``reduce`` (the reference's Thrust demo, cu:1019-1032) is not part of the Schulze
path and is not provided.
"""
from scalingelections_b200.api import (  # noqa: F401
    build_pairwise_preferences,
    compute_strongest_paths,
    get_winner_and_ranking,
    log_gpus,
    schulze,
)
