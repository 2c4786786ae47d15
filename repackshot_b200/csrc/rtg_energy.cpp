// The energy tables built into the library (generated at build time by rtg_energy_gen).
#include <cstring>

#include "rtg_tables.h"

namespace rtg {
namespace {
#include "_gen/rtg_energy_tables.inc"
template <size_t N>
std::vector<float> floats(const uint32_t (&bits)[N]) {
    std::vector<float> v(N);
    std::memcpy(v.data(), bits, N * 4);
    return v;
}
}  // namespace

const EnergyData& energy_data() {
    static const EnergyData d = {
        std::vector<uint16_t>(std::begin(E_ALBEDO), std::end(E_ALBEDO)),
        std::vector<uint16_t>(std::begin(E_SCHLICK), std::end(E_SCHLICK)),
        std::vector<uint16_t>(std::begin(E_CLEAR_IN), std::end(E_CLEAR_IN)),
        std::vector<uint16_t>(std::begin(E_CLEAR_OUT), std::end(E_CLEAR_OUT)),
        floats(E_ALBEDO_AVG),
        floats(E_SCHLICK_AVG),
    };
    return d;
}

}  // namespace rtg
