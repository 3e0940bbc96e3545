"""lakde_b200: the variational-inference hot path of falkaer/lakde's locally
adaptive KDEs on NVIDIA B200 (sm_100a).

    from lakde_b200 import LocalKNearestKDE, LocalHierarchicalKDE

The models keep the reference API (constructor arguments, fit(),
log_pred_density(), compute_elbo(), state_dict()); the custom ops keep the
reference schemas under torch.ops.lakde (see lakde_b200.kernels).  All
numerical kernels run in the in-tree CUDA library lakde_b200/_lib/liblakde_b200.so
(C ABI in include/lakde_b200.h); there is no CPU fallback.
"""

from .local_hierarchical_kde import LocalHierarchicalKDE
from .local_knn_kde import LocalKNearestKDE
from .sparse_util import PairPattern

__all__ = ["LocalKNearestKDE", "LocalHierarchicalKDE", "PairPattern"]
