// FusedConfig table entry of split configuration S(N, CL, EB, K2A, K2B)
// (configs.h, split_kernel.cuh): one job per cluster, so both schedules run
// the same direct launch; the forward with the product epilogue is left to a
// cluster configuration (kern_mul null); kern_smul is the one-launch product,
// kern_sub the forward with the subtract-and-scale output, kern_comp the
// transforms over compressed twiddle tables, kern_mulspec the forward with
// the product by a resident spectrum.
#pragma once
#include "../configs.h"
#include "../split_kernel.cuh"

#define NTTB_SG(N, CL, EB, KA, KB) SplitGeo<N, CL, EB, KA, KB>
#define NTTB_SK(N, CL, EB, KA, KB, F, A) (const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), F, A>
#define NTTB_SKC(N, CL, EB, KA, KB, F, A) \
    (const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), F, A, kOutPlain, true>
#define NTTB_SPLIT_ENTRY(N, CL, EB, KA, KB)                                                     \
    {N, CL, EB, EB, EB, KA, 1, NTTB_SG(N, CL, EB, KA, KB)::THREADS,                              \
     NTTB_SG(N, CL, EB, KA, KB)::SMEM_BYTES, NTTB_SG(N, CL, EB, KA, KB)::SMEM_BYTES,            \
     {{{NTTB_SK(N, CL, EB, KA, KB, false, Lazy4), NTTB_SK(N, CL, EB, KA, KB, false, Lazy2)},     \
       {NTTB_SK(N, CL, EB, KA, KB, true, Lazy4), NTTB_SK(N, CL, EB, KA, KB, true, Lazy2)}},      \
      {{NTTB_SK(N, CL, EB, KA, KB, false, Lazy4), NTTB_SK(N, CL, EB, KA, KB, false, Lazy2)},     \
       {NTTB_SK(N, CL, EB, KA, KB, true, Lazy4), NTTB_SK(N, CL, EB, KA, KB, true, Lazy2)}}},     \
     {nullptr, nullptr}, 1, KB,                                                                  \
     {(const void*)&split_mul_kernel<NTTB_SG(N, CL, EB, KA, KB), Lazy4>,                         \
      (const void*)&split_mul_kernel<NTTB_SG(N, CL, EB, KA, KB), Lazy2>},                        \
     SplitMulGeo<NTTB_SG(N, CL, EB, KA, KB)>::SMEM_BYTES,                                     \
     {(const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), true, Lazy4, kOutSubScale>,         \
      (const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), true, Lazy2, kOutSubScale>},        \
     {{NTTB_SKC(N, CL, EB, KA, KB, false, Lazy4), NTTB_SKC(N, CL, EB, KA, KB, false, Lazy2)},     \
      {NTTB_SKC(N, CL, EB, KA, KB, true, Lazy4), NTTB_SKC(N, CL, EB, KA, KB, true, Lazy2)}},    \
     {(const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), true, Lazy4, kOutMulSpec>,          \
      (const void*)&split_kernel<NTTB_SG(N, CL, EB, KA, KB), true, Lazy2, kOutMulSpec>}},
