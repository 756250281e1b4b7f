"""Drop-in ``scaling_elections`` module: the native-module surface that the reference's
``scaling_elections.py`` imports (scaling_elections.cu:991-1039, imported at py:30-31),
served by the sm_100a kernels of ``scalingelections_b200``.

A script run as ``python scaling_elections.py`` has its own directory first on ``sys.path``,
where its own ``scaling_elections.py`` would shadow any ``scaling_elections`` later on the
path. So either place this package directory next to the script (a package directory wins
over a same-named ``.py`` module in the same directory), or run the script through
``python -m scalingelections_b200.cli --reference-script scaling_elections.py ...``, which binds
this module in ``sys.modules`` first. ``reduce`` (the reference's Thrust demo, cu:1019-1032)
is not part of the Schulze path and is not provided.
"""
from scalingelections_b200.api import (  # noqa: F401
    build_pairwise_preferences,
    compute_strongest_paths,
    get_winner_and_ranking,
    log_gpus,
    schulze,
)
