// Host-built tables the kernels read: the Sobol generator matrices and the energy tables.
#pragma once
#include <cstdint>
#include <vector>

#include "rtg_bsdf.cuh"

namespace rtg {

void build_sobol_table(SobolTable& t);

// The six multiple-scattering tables (bsdf/energy.rs:96-300 recipe): u16 albedo[1024],
// schlick[1024], clear_in[17408], clear_out[17408]; f32 albedo_avg[32], schlick_avg[32].
struct EnergyData {
    std::vector<uint16_t> albedo, schlick, clear_in, clear_out;
    std::vector<float> albedo_avg, schlick_avg;
};
// The tables as built into the library (generated by rtg_energy_gen at build time).
const EnergyData& energy_data();

// The inverse CDF of the Blackman-Harris pixel filter (pixel_filter.rs:56-138): 256 points, in
// pixels from the centre, at u = q(i / 255) (q(s) = 2 s^2 below one half, 1 - 2 (1 - s)^2 above).
const float* blackman_harris_table();

}  // namespace rtg
