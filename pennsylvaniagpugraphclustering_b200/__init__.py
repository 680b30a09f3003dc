"""B200-native (sm_100a) implementation of the PGGC clustering hot path.

The hot path -- degree-bucket ordering, the local-move sweep, hashed
contraction, Leiden refinement and the multilevel V-cycles that drive them --
is hand-written CUDA in ``csrc/`` behind the C ABI of ``include/pggc.h``.
:mod:`.api` mirrors the reference's host interface on top of that ABI.
"""
from .api import (NEW_PART, NO_MOVE, NULL_PART, OBJECTIVES, batch_autotune, batch_run, build_coarse_graph, cluster_data,
                  clustering_methods, cut_signature, graph_from_edges, intersect_clusters, load_graph, load_view, meme_cluster,
                  coarsen_leidenR, constant_potts, generate_orderings, get_objective, local_move, local_move_strict,
                  memory_store, modularity, normalized_lcc, run_clustering, select_pass, tune_get, tune_set,
                  verify_objective, weighted_graph, write_part)
from ._lib import (METHOD_LEIDEN, METHOD_LEIDEN_PLUS, METHOD_LOUVAIN, OBJ_CPM, OBJ_LCC, OBJ_MOD, OBJ_NLCC, OBJ_WMOD,
                   DeviceError, InvalidArgument, PggcError)

__all__ = [
    "memory_store", "weighted_graph", "cluster_data", "modularity", "constant_potts", "normalized_lcc",
    "get_objective", "clustering_methods", "generate_orderings", "local_move", "local_move_strict", "select_pass",
    "build_coarse_graph", "coarsen_leidenR", "verify_objective", "run_clustering", "OBJECTIVES", "NULL_PART",
    "NO_MOVE", "NEW_PART", "METHOD_LOUVAIN", "METHOD_LEIDEN", "METHOD_LEIDEN_PLUS", "OBJ_MOD", "OBJ_WMOD",
    "OBJ_CPM", "OBJ_NLCC", "OBJ_LCC", "PggcError", "InvalidArgument", "DeviceError", "batch_run", "meme_cluster",
    "intersect_clusters", "cut_signature", "load_graph", "graph_from_edges",
    "load_view", "write_part", "batch_autotune", "tune_get", "tune_set",
]
