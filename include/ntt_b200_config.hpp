// C++ drop-in spellings of the reference's configuration header and
// launchers, on top of the C ABI in ntt_b200.h.
//
//   src/ntt_config.h:25-29     VersionConfig
//   src/ntt_config.h:31-73     PhaseLaunchConfig / NTTLaunchConfig /
//                              DefaultNTTLaunchConfig<LogN>
//   src/ntt_config.h:75-107    default_moduli / make_version_config /
//                              default_ntt_config
//   src/v04_montgomery.cu:603-658  launch_ntt<LC> / launch_intt<LC>
//
// ModulusConfig, PhaseConfig and TransformConfig are the C structs of
// ntt_b200.h (same field names and order).  A program written against the
// reference switches by including this header instead of ntt_config.h,
// dropping its own kernels and linking libntt_b200.so; its
// launch_ntt<LC>(...) / launch_intt<LC>(...) calls keep their arguments.
// The launchers return an ntt_status_t (the reference's return void; callers
// that ignore the value compile unchanged).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "ntt_b200.h"

struct VersionConfig {
    int logN;
    std::vector<ModulusConfig> moduli;
    TransformConfig transform;
};

template <int RadixStages, int StageMerging, int WarpBatching>
struct PhaseLaunchConfig {
    static constexpr int radix_stages = RadixStages;
    static constexpr int stage_merging = StageMerging;
    static constexpr int warp_batching = WarpBatching;
    static constexpr PhaseConfig runtime() { return {RadixStages, StageMerging, WarpBatching}; }
};

template <int LogN, typename NttPhase1Config, typename NttPhase2Config,
          typename InttPhase1Config, typename InttPhase2Config>
struct NTTLaunchConfig {
    static constexpr int logN = LogN;
    using NttPhase1 = NttPhase1Config;
    using NttPhase2 = NttPhase2Config;
    using InttPhase1 = InttPhase1Config;
    using InttPhase2 = InttPhase2Config;
    static constexpr TransformConfig runtime_transform() {
        return {NttPhase1::runtime(), NttPhase2::runtime(), InttPhase1::runtime(),
                InttPhase2::runtime()};
    }
};

// Same phase split as the reference's default (column phase LogN-9 stages,
// or 7 at LogN 16; row phase 9 stages).
template <int LogN>
struct DefaultNTTLaunchConfig
    : NTTLaunchConfig<LogN, PhaseLaunchConfig<(LogN == 16 ? 7 : LogN - 9), (LogN == 16 ? 4 : 3), 4>,
                      PhaseLaunchConfig<9, 3, 0>, PhaseLaunchConfig<9, 3, 0>,
                      PhaseLaunchConfig<(LogN == 16 ? 7 : LogN - 9), (LogN == 16 ? 4 : 3), 4>> {
    static_assert(LogN >= 10, "default launch config requires logN >= 10");
};

inline std::vector<ModulusConfig> default_moduli() {
    std::vector<ModulusConfig> v((size_t)ntt_default_moduli(nullptr, 0));
    ntt_default_moduli(v.data(), (int)v.size());
    return v;
}

template <typename LaunchConfig>
inline VersionConfig make_version_config() {
    return {LaunchConfig::logN, default_moduli(), LaunchConfig::runtime_transform()};
}

inline VersionConfig default_ntt_config() {
    return make_version_config<DefaultNTTLaunchConfig<16>>();
}

// launch_ntt<LC>: in place on caller-owned device buffers, the reference's
// Montgomery-form twiddle table, legacy default stream.
template <typename LaunchConfig>
inline ntt_status_t launch_ntt(uint32_t* A_dev, const uint32_t* twiddle_dev,
                               const uint32_t* moduli_dev, const uint32_t* q_inv_dev,
                               const uint32_t* r2_dev, size_t limb_count) {
    const PhaseConfig p1 = LaunchConfig::NttPhase1::runtime();
    const PhaseConfig p2 = LaunchConfig::NttPhase2::runtime();
    return ntt_launch_ntt(A_dev, twiddle_dev, moduli_dev, q_inv_dev, r2_dev, limb_count,
                          LaunchConfig::logN, &p1, &p2);
}

template <typename LaunchConfig>
inline ntt_status_t launch_intt(uint32_t* A_dev, const uint32_t* inv_twiddle_dev,
                                const uint32_t* moduli_dev, const uint32_t* q_inv_dev,
                                const uint32_t* degree_inv_dev, size_t limb_count) {
    const PhaseConfig p1 = LaunchConfig::InttPhase1::runtime();
    const PhaseConfig p2 = LaunchConfig::InttPhase2::runtime();
    return ntt_launch_intt(A_dev, inv_twiddle_dev, moduli_dev, q_inv_dev, degree_inv_dev,
                           limb_count, LaunchConfig::logN, &p1, &p2);
}
