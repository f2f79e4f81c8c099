// The mixed-precision fused E-step (estep_tc.cuh) in its 2-warpgroup shapes
// (32-sample tiles, 2 or 3 x stages), compiled apart from the default shape.
#include "estep_tc.cuh"

namespace amica {

int tc_wg2_max_clusters(int n, int m, int M, int nst) {
    return nst == 3 ? tc_max_clusters_shape<2, 3>(n, m, M) : tc_max_clusters_shape<2, 2>(n, m, M);
}

cudaError_t tc_wg2_launch(const EStepArgs& a, int nclusters, cudaStream_t st, int split, int nst) {
    return nst == 3 ? launch_tc_shape<2, 3>(a, nclusters, st, split) : launch_tc_shape<2, 2>(a, nclusters, st, split);
}

}  // namespace amica
