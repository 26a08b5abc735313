// The drop-in header's host force functions (accumulate_gravity_forces,
// accumulate_constant_pole_attraction_forces, accumulate_simple_drag_forces
// through Device_forces) on points read from a file, for comparison with the
// reference's own functions (emerald/sph2d_box/forces.cpp:63-111).
//
//   forces_host <in.bin> <out.bin>
//
// in.bin: uint64 n, uint64 terms, float mass, then terms x (int32 kind,
// float a, b, c), then n positions and n velocities (float pairs), then n
// starting forces. out.bin: the n forces after the terms.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "emerald_sph.hpp"

struct V2f {
    float x, y;
};

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    uint64_t n = 0, nt = 0;
    float mass = 0.0f;
    if (std::fread(&n, 8, 1, in) != 1 || std::fread(&nt, 8, 1, in) != 1 ||
        std::fread(&mass, 4, 1, in) != 1) {
        return 4;
    }
    emerald_b200::sph2d_box::Device_forces forces{};
    forces.terms.resize(nt);
    if (std::fread(forces.terms.data(), sizeof(emerald_force_term), nt, in) != nt) return 4;
    std::vector<V2f> x(n), v(n), f(n);
    if (std::fread(x.data(), 8, n, in) != n || std::fread(v.data(), 8, n, in) != n ||
        std::fread(f.data(), 8, n, in) != n) {
        return 4;
    }
    std::fclose(in);
    forces(n, 0.0f, 0.0f, mass, 0.0f, f.data(), x.data(), v.data());
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 3;
    std::fwrite(f.data(), 8, n, out);
    std::fclose(out);
    return 0;
}
