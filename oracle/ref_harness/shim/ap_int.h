/*
 * Minimal host-side stand-in for the Xilinx ap_int.h arbitrary-precision
 * unsigned integer, written for this project so the reference HLS kernel
 * headers compile as plain C++ (test infrastructure only).
 *
 * Supports exactly what the Falcon v1.3 kernel headers use: ap_uint<N> for
 * N <= 512, construction from integers and from bit ranges, .range(hi, lo)
 * as rvalue and as assignable proxy, wrap-around *=, ^=, >>, and implicit
 * conversion to an integer.  Storage is little-endian 64-bit words so that
 * ap_uint<32> can be reinterpreted as a float and ap_uint<512> as 64 bytes.
 */
#pragma once
#include <cstdint>
#include <cstring>

template <int N> struct ap_uint;

/* A view of bits [lo, hi] of some word array. */
struct ap_range_ref {
    uint64_t *w;
    int hi, lo;
    uint64_t get() const {
        uint64_t v = 0;
        for (int b = lo; b <= hi; b++)
            if ((w[b >> 6] >> (b & 63)) & 1ull) v |= 1ull << (b - lo);
        return v;
    }
    ap_range_ref &operator=(uint64_t v) {
        for (int b = lo; b <= hi; b++) {
            uint64_t bit = (v >> (b - lo)) & 1ull;
            w[b >> 6] = (w[b >> 6] & ~(1ull << (b & 63))) | (bit << (b & 63));
        }
        return *this;
    }
    ap_range_ref &operator=(const ap_range_ref &o) { return *this = o.get(); }
    operator uint64_t() const { return get(); }
};

template <int N>
struct ap_uint {
    static constexpr int W = (N + 63) / 64;
    uint64_t w[W];

    static uint64_t top_mask() { return (N % 64 == 0) ? ~0ull : ((1ull << (N % 64)) - 1ull); }
    void set_u64(uint64_t v) {
        std::memset(w, 0, sizeof(w));
        w[0] = v;
        w[W - 1] &= top_mask();
    }

    ap_uint() { std::memset(w, 0, sizeof(w)); }
    ap_uint(int v) { set_u64((uint64_t)(int64_t)v); }
    ap_uint(unsigned v) { set_u64(v); }
    ap_uint(long v) { set_u64((uint64_t)v); }
    ap_uint(unsigned long v) { set_u64(v); }
    ap_uint(long long v) { set_u64((uint64_t)v); }
    ap_uint(unsigned long long v) { set_u64(v); }
    ap_uint(bool v) { set_u64(v ? 1 : 0); }
    ap_uint(const ap_range_ref &r) { set_u64(r.get()); }
    template <int M> ap_uint(const ap_uint<M> &o) {
        std::memset(w, 0, sizeof(w));
        for (int i = 0; i < W && i < ap_uint<M>::W; i++) w[i] = o.w[i];
        w[W - 1] &= top_mask();
    }

    ap_range_ref range(int hi, int lo) { return ap_range_ref{w, hi, lo}; }
    uint64_t range(int hi, int lo) const {
        ap_range_ref r{const_cast<uint64_t *>(w), hi, lo};
        return r.get();
    }

    operator unsigned long long() const { return w[0]; }

    ap_uint &operator*=(uint64_t m) { set_u64(w[0] * m); return *this; }
    ap_uint &operator^=(uint64_t m) { set_u64(w[0] ^ m); return *this; }
};
