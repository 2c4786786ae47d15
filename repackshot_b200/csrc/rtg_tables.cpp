// Sobol generator matrices of the sampler (engine/crates/rt-core/src/sampler.rs:83-290): the
// logical -> Sobol dimension layout and the direction numbers of S. Joe and F. Y. Kuo,
// new-joe-kuo-6.21201 (dimensions 2..64), expanded with the Bratley–Fox recurrence. The layout
// and the direction numbers must equal the reference's for the random numbers to match.
//
// Direction numbers: https://web.maths.unsw.edu.au/~fkuo/sobol/, under this licence:
//
//   Copyright (c) 2008, Frances Y. Kuo and Stephen Joe
//   All rights reserved.
//
//   Redistribution and use in source and binary forms, with or without modification, are
//   permitted provided that the following conditions are met:
//     * Redistributions of source code must retain the above copyright notice, this list of
//       conditions and the following disclaimer.
//     * Redistributions in binary form must reproduce the above copyright notice, this list of
//       conditions and the following disclaimer in the documentation and/or other materials
//       provided with the distribution.
//     * Neither the names of the copyright holders nor the names of the University of New South
//       Wales and the University of Waikato and its contributors may be used to endorse or
//       promote products derived from this software without specific prior written permission.
//
//   THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS ``AS IS'' AND ANY EXPRESS OR IMPLIED
//   WARRANTIES, INCLUDING, BUT NOT LIMITED TO, THE IMPLIED WARRANTIES OF MERCHANTABILITY AND
//   FITNESS FOR A PARTICULAR PURPOSE ARE DISCLAIMED. IN NO EVENT SHALL THE COPYRIGHT HOLDERS BE
//   LIABLE FOR ANY DIRECT, INDIRECT, INCIDENTAL, SPECIAL, EXEMPLARY, OR CONSEQUENTIAL DAMAGES
//   (INCLUDING, BUT NOT LIMITED TO, PROCUREMENT OF SUBSTITUTE GOODS OR SERVICES; LOSS OF USE,
//   DATA, OR PROFITS; OR BUSINESS INTERRUPTION) HOWEVER CAUSED AND ON ANY THEORY OF LIABILITY,
//   WHETHER IN CONTRACT, STRICT LIABILITY, OR TORT (INCLUDING NEGLIGENCE OR OTHERWISE) ARISING IN
//   ANY WAY OUT OF THE USE OF THIS SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
#include "rtg_tables.h"

#include <cmath>

namespace rtg {

namespace {
struct DirectionNumbers { uint32_t s, a, m[9]; };
const DirectionNumbers JK[63] = {
    {1, 0, {1, 0, 0, 0, 0, 0, 0, 0, 0}},
    {2, 1, {1, 3, 0, 0, 0, 0, 0, 0, 0}},
    {3, 1, {1, 3, 1, 0, 0, 0, 0, 0, 0}},
    {3, 2, {1, 1, 1, 0, 0, 0, 0, 0, 0}},
    {4, 1, {1, 1, 3, 3, 0, 0, 0, 0, 0}},
    {4, 4, {1, 3, 5, 13, 0, 0, 0, 0, 0}},
    {5, 2, {1, 1, 5, 5, 17, 0, 0, 0, 0}},
    {5, 4, {1, 1, 5, 5, 5, 0, 0, 0, 0}},
    {5, 7, {1, 1, 7, 11, 19, 0, 0, 0, 0}},
    {5, 11, {1, 1, 5, 1, 1, 0, 0, 0, 0}},
    {5, 13, {1, 1, 1, 3, 11, 0, 0, 0, 0}},
    {5, 14, {1, 3, 5, 5, 31, 0, 0, 0, 0}},
    {6, 1, {1, 3, 3, 9, 7, 49, 0, 0, 0}},
    {6, 13, {1, 1, 1, 15, 21, 21, 0, 0, 0}},
    {6, 16, {1, 3, 1, 13, 27, 49, 0, 0, 0}},
    {6, 19, {1, 1, 1, 15, 7, 5, 0, 0, 0}},
    {6, 22, {1, 3, 1, 15, 13, 25, 0, 0, 0}},
    {6, 25, {1, 1, 5, 5, 19, 61, 0, 0, 0}},
    {7, 1, {1, 3, 7, 11, 23, 15, 103, 0, 0}},
    {7, 4, {1, 3, 7, 13, 13, 15, 69, 0, 0}},
    {7, 7, {1, 1, 3, 13, 7, 35, 63, 0, 0}},
    {7, 8, {1, 3, 5, 9, 1, 25, 53, 0, 0}},
    {7, 14, {1, 3, 1, 13, 9, 35, 107, 0, 0}},
    {7, 19, {1, 3, 1, 5, 27, 61, 31, 0, 0}},
    {7, 21, {1, 1, 5, 11, 19, 41, 61, 0, 0}},
    {7, 28, {1, 3, 5, 3, 3, 13, 69, 0, 0}},
    {7, 31, {1, 1, 7, 13, 1, 19, 1, 0, 0}},
    {7, 32, {1, 3, 7, 5, 13, 19, 59, 0, 0}},
    {7, 37, {1, 1, 3, 9, 25, 29, 41, 0, 0}},
    {7, 41, {1, 3, 5, 13, 23, 1, 55, 0, 0}},
    {7, 42, {1, 3, 7, 3, 13, 59, 17, 0, 0}},
    {7, 50, {1, 3, 1, 3, 5, 53, 69, 0, 0}},
    {7, 55, {1, 1, 5, 5, 23, 33, 13, 0, 0}},
    {7, 56, {1, 1, 7, 7, 1, 61, 123, 0, 0}},
    {7, 59, {1, 1, 7, 9, 13, 61, 49, 0, 0}},
    {7, 62, {1, 3, 3, 5, 3, 55, 33, 0, 0}},
    {8, 14, {1, 3, 1, 15, 31, 13, 49, 245, 0}},
    {8, 21, {1, 3, 5, 15, 31, 59, 63, 97, 0}},
    {8, 22, {1, 3, 1, 11, 11, 11, 77, 249, 0}},
    {8, 38, {1, 3, 1, 11, 27, 43, 71, 9, 0}},
    {8, 47, {1, 1, 7, 15, 21, 11, 81, 45, 0}},
    {8, 49, {1, 3, 7, 3, 25, 31, 65, 79, 0}},
    {8, 50, {1, 3, 1, 1, 19, 11, 3, 205, 0}},
    {8, 52, {1, 1, 5, 9, 19, 21, 29, 157, 0}},
    {8, 56, {1, 3, 7, 11, 1, 33, 89, 185, 0}},
    {8, 67, {1, 3, 3, 3, 15, 9, 79, 71, 0}},
    {8, 70, {1, 3, 7, 11, 15, 39, 119, 27, 0}},
    {8, 84, {1, 1, 3, 1, 11, 31, 97, 225, 0}},
    {8, 97, {1, 1, 1, 3, 23, 43, 57, 177, 0}},
    {8, 103, {1, 3, 7, 7, 17, 17, 37, 71, 0}},
    {8, 115, {1, 3, 1, 5, 27, 63, 123, 213, 0}},
    {8, 122, {1, 1, 3, 5, 11, 43, 53, 133, 0}},
    {9, 8, {1, 3, 5, 5, 29, 17, 47, 173, 479}},
    {9, 13, {1, 3, 3, 11, 3, 1, 109, 9, 69}},
    {9, 16, {1, 1, 1, 5, 17, 39, 23, 5, 343}},
    {9, 22, {1, 3, 1, 5, 25, 15, 31, 103, 499}},
    {9, 25, {1, 1, 1, 11, 11, 17, 63, 105, 183}},
    {9, 44, {1, 1, 5, 11, 9, 29, 97, 231, 363}},
    {9, 47, {1, 1, 5, 15, 19, 45, 41, 7, 383}},
    {9, 52, {1, 3, 7, 7, 31, 19, 83, 137, 221}},
    {9, 55, {1, 1, 1, 3, 23, 15, 111, 223, 83}},
    {9, 59, {1, 1, 5, 13, 31, 15, 55, 25, 161}},
    {9, 62, {1, 1, 3, 13, 25, 47, 39, 87, 257}},
};
// sampler.rs:83: camera x/y, lens u/v, then per vertex light select, light u/v, bsdf u/v, roulette.
const uint8_t LAYOUT[64] = {0,  1,  11, 50, 19, 2,  15, 10, 13, 20, 21, 5,  27, 3,  59, 25, 26, 6,  57, 18, 47, 28,
                            31, 24, 44, 22, 58, 34, 37, 49, 52, 4,  9,  39, 41, 7,  12, 16, 29, 42, 45, 8,  38, 14,
                            46, 48, 51, 33, 36, 32, 56, 53, 54, 35, 63, 43, 62, 55, 60, 23, 30, 17, 40, 61};
}  // namespace

void build_sobol_table(SobolTable& t) {
    for (int k = 0; k < 32; ++k) t.m[0][k] = 1u << (31 - k);
    for (int d = 1; d < 64; ++d) {
        const DirectionNumbers& jk = JK[d - 1];
        uint32_t* v = t.m[d];
        for (uint32_t i = 0; i < 32; ++i) {
            if (i < jk.s) {
                v[i] = jk.m[i] << (31 - i);
            } else {
                uint32_t value = v[i - jk.s] ^ (v[i - jk.s] >> jk.s);
                for (uint32_t k = 1; k < jk.s; ++k)
                    if ((jk.a >> (jk.s - 1 - k)) & 1u) value ^= v[i - k];
                v[i] = value;
            }
        }
    }
    for (int i = 0; i < 64; ++i) t.layout[i] = LAYOUT[i];
}

// The window of F. J. Harris (Proc. IEEE 66, 1978), a0 - a1 cos 2 pi t + a2 cos 4 pi t - a3 cos 6 pi t,
// three pixels wide: each point of the table by 100 bisections of its integral in double, rounded
// to float, as the reference makes its table.
const float* blackman_harris_table() {
    static float table[256];
    static bool ready = false;
    if (ready) return table;
    const double a0 = 0.35875, a1 = 0.48829, a2 = 0.14128, a3 = 0.01168, radius = 1.5;
    const double two_pi = 2.0 * 3.14159265358979323846;
    auto integral = [&](double x) {  // of the normalised window, from its left end to x pixels
        double t = (x + radius) / (2.0 * radius);
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        return (a0 * t - a1 * std::sin(two_pi * t) / two_pi + a2 * std::sin(2.0 * two_pi * t) / (2.0 * two_pi) -
                a3 * std::sin(3.0 * two_pi * t) / (3.0 * two_pi)) /
               a0;
    };
    for (int i = 0; i < 256; ++i) {
        const double s = (double)i / 255.0;
        const double u = s < 0.5 ? 2.0 * s * s : 1.0 - 2.0 * (1.0 - s) * (1.0 - s);
        double lo = -radius, hi = radius;
        for (int k = 0; k < 100; ++k) {
            const double mid = 0.5 * (lo + hi);
            if (integral(mid) < u) lo = mid;
            else hi = mid;
        }
        table[i] = (float)(0.5 * (lo + hi));
    }
    ready = true;
    return table;
}

}  // namespace rtg
