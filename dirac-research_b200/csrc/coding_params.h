// Per-picture coding parameters the reference encoder derives on the host: the lambdas of
// EncoderParams::CalcLambdas (libdirac_common/common.cpp:451-476) and
// PictureCompressor::GetCompLambda (libdirac_encoder/picture_compress.cpp:532-580), the
// perceptual-weight scale of PictureCompressor::CodeResidue (picture_compress.cpp:418-428) and
// the initial factors of EntropyCorrector::Init (common.cpp:79-131).  Shared by the sequence
// encoder and the picture batch.
#pragma once

#include <algorithm>
#include <cmath>

namespace dgpu {

struct Lambdas {
    float i, l1, l2, me;
};

// EncoderParams::CalcLambdas: float members, std::sqrt of a float member.
inline Lambdas calc_lambdas(float qf) {
    Lambdas L;
    L.i = (float)(std::pow(10.0, (12.0 - (double)qf) / 2.5) / 16.0);
    L.l1 = (float)((double)L.i * 4.0);
    L.l2 = (float)((double)L.i * 32.0);
    L.me = (float)((double)std::sqrt(L.l1) * 2.0);
    return L;
}

// GetCompLambda: std::log10 of the float lambdas is the single-precision overload; the blend
// is double; U and V factors 1.5 / 0.75 (libdirac_encoder/dirac_encoder.cpp:552-553)
// multiply in float.
inline float component_lambda(const Lambdas& L, bool intra, bool is_b, double intra_ratio, int comp) {
    float lambda;
    if (intra) {
        lambda = L.i;
    } else {
        const double log_intra = std::log10(L.i);
        const double log_pic = is_b ? std::log10(L.l2) : std::log10(L.l1);
        const float ir = (float)intra_ratio;
        lambda = (float)std::pow(10.0, 3.0 * ir * log_intra + (1.0 - 3.0 * ir) * log_pic);
    }
    if (comp == 1) lambda *= 1.5f;
    if (comp == 2) lambda *= 0.75f;
    return lambda;
}

// CodeResidue's cycles-per-degree scale of an inter picture (1 for intra).
inline double perceptual_scale(bool intra, double intra_ratio) {
    if (intra) return 1.0;
    const float ir = (float)intra_ratio;
    const double s = 5.0 * ir * 1.0 + (1.0 - 5.0 * ir) * 0.125;
    return std::max(0.125, std::min(1.2, s));
}

// EntropyCorrector::Init: the same initial factors for all components.
inline void initial_ecf(int depth, bool intra, float* out) {
    const int nb = 3 * depth + 1;
    for (int b = 0; b < nb; ++b) out[b] = 0.75f;
    for (int b = nb - 4; b < nb - 1; ++b) out[b] = intra ? 0.85f : 0.75f;
    out[nb - 1] = intra ? 1.0f : 0.85f;
}

}  // namespace dgpu
