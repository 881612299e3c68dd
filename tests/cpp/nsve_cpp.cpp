// Drives the C++ mirror (include/bfps_b200.hpp) the way NSVEparticles does:
// reads an initial vorticity (reference complex layout) and tracer
// positions from a binary file, sets the physical members, runs K
// NSVEparticles steps and writes the final vorticity, tracer state and the
// sampled acceleration; with a ninth argument "ensemble" the steps go
// through a one-member ensemble.
//   nsve_cpp <precision 4|8> <n> <ntracers> <steps> <dt> <in> <out> [ensemble]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "bfps_b200.hpp"

template <typename rnumber>
static int run(int n, long long nt, int steps, double dt, const char* in, const char* out,
               bool ens) {
    using cnumber = std::complex<rnumber>;
    bfps_b200::vorticity_equation<rnumber> fs("cpp_test", n, n, n);
    fs.nu = 0.05;
    std::snprintf(fs.forcing_type, sizeof(fs.forcing_type), "linear");
    fs.famplitude = 0.5;
    fs.fk0 = 1.5;
    fs.fk1 = 3.0;
    std::vector<cnumber> w(fs.complex_size());
    std::vector<double> pos(3 * nt);
    FILE* f = std::fopen(in, "rb");
    if (!f) return 2;
    if (std::fread(w.data(), sizeof(cnumber), w.size(), f) != w.size() ||
        std::fread(pos.data(), sizeof(double), pos.size(), f) != pos.size())
        return 3;
    std::fclose(f);
    fs.io_checkpoint_read(w.data(), 0);
    bfps_b200::particles_system ps(fs, nt, 2, 1, 3, pos.data(), nullptr, nullptr, 1);
    if (ens) {
        bfps_b200::ensemble e;
        e.add(fs, dt, &ps);
        e.step(steps);
        while (!e.wait(1000.0)) {
        }
        if (e.count() != 1 || !(e.last_ms() > 0)) return 6;
        e.remove(fs);
    } else {
        for (int s = 0; s < steps; ++s) bfps_b200::NSVEparticles_step(fs, ps, dt);
    }
    std::vector<double> state(3 * nt), rhs(3 * 3 * nt), acc(3 * nt);
    fs.get_cvorticity(w.data());
    ps.get_state(state.data(), rhs.data(), nullptr);
    ps.sample_acceleration(acc.data());
    f = std::fopen(out, "wb");
    if (!f) return 4;
    std::fwrite(&fs.iteration, sizeof(int), 1, f);
    const int sidx = ps.get_step_idx();
    std::fwrite(&sidx, sizeof(int), 1, f);
    std::fwrite(w.data(), sizeof(cnumber), w.size(), f);
    std::fwrite(state.data(), sizeof(double), state.size(), f);
    std::fwrite(rhs.data(), sizeof(double), rhs.size(), f);
    std::fwrite(acc.data(), sizeof(double), acc.size(), f);
    std::fclose(f);
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 8 && argc != 9) return 1;
    const bool ens = argc == 9 && std::string(argv[8]) == "ensemble";
    try {
        const int prec = std::atoi(argv[1]);
        const int n = std::atoi(argv[2]);
        const long long nt = std::atoll(argv[3]);
        const int steps = std::atoi(argv[4]);
        const double dt = std::atof(argv[5]);
        return prec == 4 ? run<float>(n, nt, steps, dt, argv[6], argv[7], ens)
                         : run<double>(n, nt, steps, dt, argv[6], argv[7], ens);
    } catch (const bfps_b200::error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 5;
    }
}
