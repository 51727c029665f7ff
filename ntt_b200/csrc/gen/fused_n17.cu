// Instantiations of the fused kernel for logN = 17 (see configs.h).
#include "../configs.h"
#include "../fused_kernel.cuh"

namespace nttb {
#define NTTB_G(N, CL, R1, EB, K1A, K2A) Geometry<N, CL, R1, EB, K1A, K2A>
#define NTTB_K(N, CL, R1, EB, K1A, K2A, F, S, A) \
    (const void*)&fused_kernel<NTTB_G(N, CL, R1, EB, K1A, K2A), F, S, A>
#define NTTB_ENTRY(N, CL, R1, EB, K1A, K2A)                                                   \
    {N, CL, R1, EB, K1A, K2A, NTTB_G(N, CL, R1, EB, K1A, K2A)::THREADS,                      \
     NTTB_G(N, CL, R1, EB, K1A, K2A)::SMEM_BYTES,                                            \
     NTTB_G(N, CL, R1, EB, K1A, K2A)::SMEM_BYTES_DIRECT,                                     \
     {{{NTTB_K(N, CL, R1, EB, K1A, K2A, false, false, Lazy4),                                \
        NTTB_K(N, CL, R1, EB, K1A, K2A, false, false, Lazy2)},                               \
       {NTTB_K(N, CL, R1, EB, K1A, K2A, true, false, Lazy4),                                 \
        NTTB_K(N, CL, R1, EB, K1A, K2A, true, false, Lazy2)}},                               \
      {{NTTB_K(N, CL, R1, EB, K1A, K2A, false, true, Lazy4),                                 \
        NTTB_K(N, CL, R1, EB, K1A, K2A, false, true, Lazy2)},                                \
       {NTTB_K(N, CL, R1, EB, K1A, K2A, true, true, Lazy4),                                  \
        NTTB_K(N, CL, R1, EB, K1A, K2A, true, true, Lazy2)}}}},
extern const FusedConfig kFusedN17[] = {NTTB_CFG_N17(NTTB_ENTRY)};
extern const int kFusedN17Count = sizeof(kFusedN17) / sizeof(kFusedN17[0]);
}  // namespace nttb
