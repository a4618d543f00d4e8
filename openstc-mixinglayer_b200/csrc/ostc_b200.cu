// ostc_b200.cu -- the library's one CUDA translation unit: sm_100a kernels of the RHS + SSP-RK3 path
// (air and mixtures), their launch machinery and the C ABI (include/ostc.h).
//
// One translation unit on purpose: the mixture tables live in __constant__ memory (c_mix), and
// without relocatable device code every translation unit would get its own copy, so every kernel
// and every launch is compiled here.  The parts, in include order:
//   dev_types.cuh    device views of blocks, states, faces and interfaces
//   air_kernels.cuh  air fluxes, viscous + update, time step, boundary faces, interfaces, set-up
//   ostc_adj_air.cuh the air right-hand side's adjoint
//   ostc_mix.cuh, ostc_adj.cuh, ostc_stat.cuh, ostc_steady.cuh, pv_mix.cuh, ostc_df.cuh
//                    mixture kernels, adjoint, statistics, steady / DPLUR, mixture primitive
//                    reconstruction, digital-filter inflow
//   context.cuh      the ostc_ctx context and per-block resources
//   enqueue.cuh      launch helpers, stage / step enqueue, autotuner, initialisation
//   api_core.cuh, api_stat.cuh, api_step.cuh, api_plt.cuh, api_misc.cuh   the C ABI

#include "air_math.cuh"
#include "host.h"
#include "ostc.h"

#include <cuda_runtime.h>
#include <curand_kernel.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "dev_types.cuh"

#include "ostc_mix.cuh"
#include "ostc_adj.cuh"
#include "ostc_stat.cuh"
#include "ostc_steady.cuh"
#include "pv_mix.cuh"
#include "ostc_df.cuh"

static_assert(ostc::kMS <= 16, "DevFace::y holds the inflow mass fractions of at most 16 species");

#include "air_kernels.cuh"
#include "ostc_adj_air.cuh"
#include "context.cuh"
#include "enqueue.cuh"
#include "api_core.cuh"
#include "api_stat.cuh"
#include "api_step.cuh"
#include "api_plt.cuh"
#include "api_misc.cuh"
