// FusedConfig table entry of one configuration X(N, CL, R1, EB, K1A, K2A, NP)
// (configs.h): its eight kernels [staged][fwd][lazy2], the two direct
// forwards with the product epilogue [lazy2] and the two with the
// subtract-and-scale output [lazy2].  NP > 1 has no staged form, so
// its staged entries are the direct kernels (and their shared memory size).
#pragma once
#include "../configs.h"
#include "../fused_kernel.cuh"

#define NTTB_G(N, CL, R1, EB, K1A, K2A, NP) Geometry<N, CL, R1, EB, K1A, K2A, NP>
#define NTTB_K(N, CL, R1, EB, K1A, K2A, NP, F, S, A) \
    (const void*)&fused_kernel<NTTB_G(N, CL, R1, EB, K1A, K2A, NP), F, (S) && (NP) == 1, A>
#define NTTB_KM(N, CL, R1, EB, K1A, K2A, NP, A) \
    (const void*)&fused_kernel<NTTB_G(N, CL, R1, EB, K1A, K2A, NP), true, false, A, true>
#define NTTB_KSUB(N, CL, R1, EB, K1A, K2A, NP, A) \
    (const void*)&fused_kernel<NTTB_G(N, CL, R1, EB, K1A, K2A, NP), true, false, A, false, true>
#define NTTB_ENTRY(N, CL, R1, EB, K1A, K2A, NP)                                               \
    {N, CL, R1, EB, K1A, K2A, NP, NTTB_G(N, CL, R1, EB, K1A, K2A, NP)::THREADS,              \
     (NP) == 1 ? NTTB_G(N, CL, R1, EB, K1A, K2A, NP)::SMEM_BYTES                            \
               : NTTB_G(N, CL, R1, EB, K1A, K2A, NP)::SMEM_BYTES_DIRECT,                    \
     NTTB_G(N, CL, R1, EB, K1A, K2A, NP)::SMEM_BYTES_DIRECT,                                 \
     {{{NTTB_K(N, CL, R1, EB, K1A, K2A, NP, false, false, Lazy4),                            \
        NTTB_K(N, CL, R1, EB, K1A, K2A, NP, false, false, Lazy2)},                           \
       {NTTB_K(N, CL, R1, EB, K1A, K2A, NP, true, false, Lazy4),                             \
        NTTB_K(N, CL, R1, EB, K1A, K2A, NP, true, false, Lazy2)}},                           \
      {{NTTB_K(N, CL, R1, EB, K1A, K2A, NP, false, true, Lazy4),                             \
        NTTB_K(N, CL, R1, EB, K1A, K2A, NP, false, true, Lazy2)},                            \
       {NTTB_K(N, CL, R1, EB, K1A, K2A, NP, true, true, Lazy4),                              \
        NTTB_K(N, CL, R1, EB, K1A, K2A, NP, true, true, Lazy2)}}},                           \
     {NTTB_KM(N, CL, R1, EB, K1A, K2A, NP, Lazy4), NTTB_KM(N, CL, R1, EB, K1A, K2A, NP, Lazy2)}, \
     0, 0, {nullptr, nullptr}, 0,                                                            \
     {NTTB_KSUB(N, CL, R1, EB, K1A, K2A, NP, Lazy4),                                          \
      NTTB_KSUB(N, CL, R1, EB, K1A, K2A, NP, Lazy2)}},
