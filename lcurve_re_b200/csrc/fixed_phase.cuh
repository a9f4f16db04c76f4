// fixed_phase.cuh — eclipse tests of the mixed sweeps in 64-bit fixed-point phase.
//
// The FP64 sweep tests a face's eclipse at phase phin with the reference's
// doubles, ecl_range (comp_light_flat.cpp:171-173). The mixed sweeps keep
// phases and ranges as 64-bit fixed-point fractions of a turn instead, so the
// test is one 64-bit subtract and compare per face and entry, and its
// decisions are the reference's: a face's flux is a noticeable part of a
// light curve when a hot, finely gridded star dominates the light (one face
// of a 200,000-face white dwarf is 2e-5 of it), so a flag that differed from
// the reference's within even 2^-32 of a boundary would show.
#ifndef LCG_FIXED_PHASE_CUH
#define LCG_FIXED_PHASE_CUH

#ifndef LCG_FX_FN
#define LCG_FX_FN __host__ __device__ __forceinline__
#endif

namespace lcg {

// phase_fx64: a phase in [0, 1] as floor(x 2^64). Exact for x >= 2^-12 (such
// doubles have no bits below 2^-64) and monotone below it; x = 1 (phi -
// floor(phi) rounds to 1 just below a whole phase) maps to 2^64 - 1, which
// orders it after every ingress and egress below 1, as the reference's
// comparisons of 1.0 do.
LCG_FX_FN unsigned long long phase_fx64(double x) {
    if (!(x < 1.0)) return ~0ull;
    if (!(x > 0.0)) return 0ull;
    const double t = x * 4294967296.0;                 // exact
    const double hi = floor(t);
    const double lo = floor((t - hi) * 4294967296.0);  // t - hi and the scaling exact
    return ((unsigned long long)hi << 32) | (unsigned long long)lo;
}

// Eclipse range [in1, out1] (ingress in [0, 1), egress in [in1, in1 + 1]) as
// (I, W + 1): I = phase_fx64(in1), W = (phase_fx64(out1 mod 1) - I) mod 2^64.
// A phase P is then visible iff (P - I) mod 2^64 >= W + 1, which is
// ecl_range's !((phin >= in && phin <= out) || phin <= out - 1)
// (comp_light_flat.cpp:171-173) decision for decision, out1 - 1 being exact
// for out1 in [1, 2]; exact but where a phase and a boundary both lie below
// 2^-12 and within 2^-64 of each other. (0, 0), the record of a face without a
// range, is never eclipsed. A range of a whole turn is (2^64 - 1, 2^64 - 1):
// visible only at P = 2^64 - 2, which no double in [0, 1] maps to.
LCG_FX_FN ulonglong2 ecl_fx64(double in1, double out1) {
    if (!(out1 - in1 < 1.0)) return make_ulonglong2(~0ull, ~0ull);  // the whole orbit
    const unsigned long long I = phase_fx64(in1);
    const unsigned long long W = phase_fx64(out1 >= 1.0 ? out1 - 1.0 : out1) - I;
    return make_ulonglong2(I, W == ~0ull ? W : W + 1);
}

}  // namespace lcg

#endif
