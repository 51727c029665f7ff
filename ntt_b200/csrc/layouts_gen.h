// GENERATED by gen_layouts.py from configs.h -- do not edit.
// Per configuration: the work-buffer bank-spreading layout (A1, C1, A2, C2,
// size in words) and the lane masks the search assumed (checked against
// PassLayout by static_assert in ntt_core.cuh).
#pragma once
#include <cstdint>

namespace nttb {

template <int N, int CL, int R1, int EB, int K1A, int K2A>
struct LayoutTable;

template <>
struct LayoutTable<10, 0, 5, 5, 5, 5> {
    static constexpr int XW[5] = {5, 4, 10, 0, 1148};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x3d0u;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<11, 0, 6, 5, 1, 5> {
    static constexpr int XW[5] = {5, 4, 11, 0, 2300};
    static constexpr uint32_t lanes_P1A = 0x1f0u;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<12, 0, 7, 5, 3, 5> {
    static constexpr int XW[5] = {5, 4, 12, 0, 4604};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x21eu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<12, 0, 6, 4, 3, 3> {
    static constexpr int XW[5] = {5, 4, 12, 0, 4604};
    static constexpr uint32_t lanes_P1A = 0x3eu;
    static constexpr uint32_t lanes_P1B = 0x3eu;
    static constexpr uint32_t lanes_P2A = 0x1c6u;
    static constexpr uint32_t lanes_P2B = 0x1f0u;
};

template <>
struct LayoutTable<13, 0, 8, 5, 3, 5> {
    static constexpr int XW[5] = {5, 4, 13, 0, 9212};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<14, 0, 9, 5, 4, 5> {
    static constexpr int XW[5] = {5, 4, 14, 0, 18428};
    static constexpr uint32_t lanes_P1A = 0x3eu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<14, 1, 9, 5, 4, 5> {
    static constexpr int XW[5] = {5, 2, 9, 16, 8942};
    static constexpr uint32_t lanes_P1A = 0x3eu;
    static constexpr uint32_t lanes_P1B = 0x20fu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<14, 1, 6, 6, 6, 4> {
    static constexpr int XW[5] = {6, 4, 13, 0, 8700};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x760u;
    static constexpr uint32_t lanes_P2A = 0x70cu;
    static constexpr uint32_t lanes_P2B = 0x7c0u;
};

template <>
struct LayoutTable<15, 1, 10, 5, 5, 5> {
    static constexpr int XW[5] = {5, 1, 10, 16, 17135};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x20fu;
    static constexpr uint32_t lanes_P2A = 0x3e0u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<15, 2, 8, 5, 3, 4> {
    static constexpr int XW[5] = {5, 4, 13, 0, 9212};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x386u;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<15, 2, 6, 6, 6, 5> {
    static constexpr int XW[5] = {6, 4, 9, 16, 8940};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x760u;
    static constexpr uint32_t lanes_P2A = 0x60eu;
    static constexpr uint32_t lanes_P2B = 0x7c0u;
};

template <>
struct LayoutTable<16, 3, 8, 5, 3, 4> {
    static constexpr int XW[5] = {5, 1, 13, 0, 8447};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x30eu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<16, 3, 7, 5, 3, 5> {
    static constexpr int XW[5] = {6, 4, 9, 16, 8940};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x3eu;
    static constexpr uint32_t lanes_P2A = 0x20fu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<16, 2, 8, 5, 3, 4> {
    static constexpr int XW[5] = {5, 4, 14, 0, 18428};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x30eu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<16, 4, 8, 5, 3, 4> {
    static constexpr int XW[5] = {6, 4, 9, 16, 4460};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x20fu;
    static constexpr uint32_t lanes_P2A = 0x30eu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<16, 3, 8, 4, 4, 4> {
    static constexpr int XW[5] = {6, 4, 13, 0, 8700};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x10fu;
    static constexpr uint32_t lanes_P2B = 0x1f0u;
};

template <>
struct LayoutTable<16, 3, 6, 6, 6, 5> {
    static constexpr int XW[5] = {6, 4, 13, 0, 8700};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x760u;
    static constexpr uint32_t lanes_P2A = 0x41eu;
    static constexpr uint32_t lanes_P2B = 0x7c0u;
};

template <>
struct LayoutTable<16, 4, 6, 6, 6, 4> {
    static constexpr int XW[5] = {5, 2, 6, 2, 4476};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x7a0u;
    static constexpr uint32_t lanes_P2A = 0x43cu;
    static constexpr uint32_t lanes_P2B = 0x7c0u;
};

template <>
struct LayoutTable<16, 4, 8, 4, 4, 4> {
    static constexpr int XW[5] = {5, 2, 12, 0, 4350};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x10fu;
    static constexpr uint32_t lanes_P2A = 0x10fu;
    static constexpr uint32_t lanes_P2B = 0x1f0u;
};

template <>
struct LayoutTable<17, 3, 8, 5, 3, 5> {
    static constexpr int XW[5] = {6, 4, 9, 16, 17900};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x20fu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<17, 4, 8, 5, 3, 5> {
    static constexpr int XW[5] = {6, 4, 9, 16, 8940};
    static constexpr uint32_t lanes_P1A = 0x7cu;
    static constexpr uint32_t lanes_P1B = 0x1fu;
    static constexpr uint32_t lanes_P2A = 0x20fu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct LayoutTable<17, 4, 6, 6, 6, 5> {
    static constexpr int XW[5] = {6, 4, 13, 0, 8700};
    static constexpr uint32_t lanes_P1A = 0x1fu;
    static constexpr uint32_t lanes_P1B = 0x760u;
    static constexpr uint32_t lanes_P2A = 0x3eu;
    static constexpr uint32_t lanes_P2B = 0x7c0u;
};

template <int N, int CL, int EB, int K2A, int K2B>
struct SplitLayoutTable;

template <>
struct SplitLayoutTable<16, 3, 5, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 8, 9460};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x386u;
    static constexpr uint32_t lanes_P2C = 0x3e0u;
};

template <>
struct SplitLayoutTable<16, 3, 4, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 16, 9708};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x10fu;
    static constexpr uint32_t lanes_P2C = 0x1f0u;
};

template <>
struct SplitLayoutTable<16, 3, 5, 3, 4> {
    static constexpr int XW[5] = {5, 4, 8, 16, 9708};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x30eu;
    static constexpr uint32_t lanes_P2C = 0x3e0u;
};

template <>
struct SplitLayoutTable<16, 4, 5, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 8, 4724};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x386u;
    static constexpr uint32_t lanes_P2C = 0x3e0u;
};

template <>
struct SplitLayoutTable<16, 4, 4, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 16, 4844};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x10fu;
    static constexpr uint32_t lanes_P2C = 0x1f0u;
};

template <>
struct SplitLayoutTable<17, 4, 5, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 16, 9708};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x30eu;
    static constexpr uint32_t lanes_P2C = 0x3e0u;
};

template <>
struct SplitLayoutTable<15, 2, 5, 5, 5> {
    static constexpr int XW[5] = {5, 4, 13, 0, 9212};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x3e0u;
};

template <>
struct SplitLayoutTable<15, 2, 4, 4, 4> {
    static constexpr int XW[5] = {5, 4, 8, 8, 9460};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x187u;
    static constexpr uint32_t lanes_P2C = 0x1f0u;
};

template <>
struct SplitLayoutTable<15, 3, 5, 4, 3> {
    static constexpr int XW[5] = {5, 4, 12, 0, 4604};
    static constexpr uint32_t lanes_P2A = 0x1fu;
    static constexpr uint32_t lanes_P2B = 0x3c4u;
    static constexpr uint32_t lanes_P2C = 0x3e0u;
};

}  // namespace nttb
