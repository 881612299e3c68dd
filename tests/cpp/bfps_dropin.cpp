// Written as bfps code is written, against the drop-in headers under
// include/bfps (field, kspace, vorticity_equation, particles_system_builder),
// in the order NSVE / NSVEparticles use them (bfps/cpp/full_code/NSVE.cpp:
// 31-135, NSVEparticles.cpp:7-98): construct the solver, fill cvorticity's
// host data and apply io_checkpoint's read-time steps, build the tracers,
// then per iteration: statistics of the vorticity and the velocity through a
// separate field (NSVE::do_stats), compute_velocity(cvorticity),
// cvelocity->ift(), completeLoop, step.  Writes the final state, tracer
// positions, the last statistics and a host-side kspace summary.
//   bfps_dropin <n> <ntracers> <steps> <dt> <in> <out>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "particles/particles_system_builder.hpp"
#include "vorticity_equation.hpp"

int main(int argc, char** argv) {
    if (argc != 7) return 1;
    const int n = std::atoi(argv[1]);
    const long long nt = std::atoll(argv[2]);
    const int steps = std::atoi(argv[3]);
    const double dt = std::atof(argv[4]);
    try {
        vorticity_equation<double, FFTW> fs("dropin", n, n, n, 1.0, 1.0, 1.0, FFTW_ESTIMATE);
        fs.nu = 0.05;
        std::snprintf(fs.forcing_type, sizeof(fs.forcing_type), "linear");
        fs.famplitude = 0.5;
        fs.fk0 = 1.5;
        fs.fk1 = 3.0;
        fs.iteration = 0;
        field<double, FFTW, THREE>* tmp_vec_field =
            new field<double, FFTW, THREE>(n, n, n, MPI_COMM_WORLD, FFTW_ESTIMATE);
        tmp_vec_field->real_space_representation = false;

        std::vector<double> pos(3 * nt);
        FILE* f = std::fopen(argv[5], "rb");
        if (!f) return 2;
        const size_t nc = 2 * fs.cvorticity->clayout->local_size;
        if (std::fread(fs.cvorticity->get_rdata(), sizeof(double), nc, f) != nc ||
            std::fread(pos.data(), sizeof(double), pos.size(), f) != pos.size())
            return 3;
        std::fclose(f);
        fs.io_checkpoint_read_host();

        auto ps = particles_system_builder<long long, double, FFTW, THREE, double>(
            fs.cvelocity, fs.kk, 3, nt, pos.data(), nullptr, 3, 2, MPI_COMM_WORLD,
            fs.iteration + 1);
        if (ps->getNbRhs() != 3 || ps->getGlobalNbParticles() != nt) return 6;

        std::vector<double> spec_w, mom_w, spec_u, mom_u;
        std::vector<int64_t> hist_w, hist_u;
        for (int s = 0; s < steps; ++s) {
            // NSVE::do_stats
            *tmp_vec_field = fs.cvorticity->get_cdata();
            tmp_vec_field->compute_stats(fs.kk, spec_w, mom_w, hist_w, 5.0 / std::sqrt(3.0), 64);
            fs.compute_velocity(fs.cvorticity);
            *tmp_vec_field = fs.cvelocity->get_cdata();
            tmp_vec_field->compute_stats(fs.kk, spec_u, mom_u, hist_u, 1.0 / std::sqrt(3.0), 64);
            // NSVEparticles::step
            fs.compute_velocity(fs.cvorticity);
            fs.cvelocity->ift();
            ps->completeLoop(dt);
            fs.step(dt);
        }
        f = std::fopen(argv[6], "wb");
        if (!f) return 4;
        int hdr[4] = {fs.iteration, ps->get_step_idx(), fs.kk->nshells, (int)hist_u.size()};
        std::fwrite(hdr, sizeof(int), 4, f);
        std::fwrite(fs.cvorticity->get_rdata(), sizeof(double), nc, f);
        std::fwrite(ps->getParticlesPositions(), sizeof(double), 3 * nt, f);
        std::fwrite(spec_u.data(), sizeof(double), spec_u.size(), f);
        std::fwrite(mom_u.data(), sizeof(double), mom_u.size(), f);
        std::fwrite(hist_u.data(), sizeof(int64_t), hist_u.size(), f);
        const double ks[3] = {fs.kk->kM, fs.kk->dk, fs.kk->dealias_filter[10]};
        std::fwrite(ks, sizeof(double), 3, f);
        std::fwrite(fs.kk->kshell.data(), sizeof(double), fs.kk->kshell.size(), f);
        std::fclose(f);
        delete tmp_vec_field;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 5;
    }
    return 0;
}
