/*
 * ref_flow — drives the REFERENCE's own Wilson-flow code (compiled from its
 * sources by oracle/Makefile against the single-rank shims in ref/shim) and
 * prints its numbers at full precision.  Test infrastructure only: it is the
 * parity anchor for the CPU restatement (oracle/ymoracle.c) and the timed
 * "reference" CPU baseline.  Nothing in the product links it.
 *
 * WilsonFlow::flowStep is private (include/Apps/wilsonflow.h:82), so the RK3
 * step below is re-spelt with the reference's PUBLIC primitives in the exact
 * order of src/Apps/wilsonflow.cpp:141-172:
 *   PureGauge::computeDerivative  (src/Actions/puregauge.cpp:62-79)
 *   exp(Lattice<SU3>)             (include/Math/lattice.h:247-261 -> src/Math/su3.cpp:96-183)
 *   Lattice * Lattice, scalar ops (include/Math/lattice.h:130-228)
 * Observables come from SuperObs::compute (src/Observables/superobs.cpp:31-128)
 * and links are read with LatticeIO::InputConf::readConf
 * (src/InputOutput/inputconf.cpp:114-155), so the .bin layout is the
 * reference's own.
 *
 * Modes (all sizes are the global lattice, one rank):
 *   flow   CONF Nx Ny Nz Nt EPS NSTEPS EVERY [OUT.bin]
 *          rows "step t plaq topc energy" (%.17g) at step 0 and every EVERY
 *          steps; t is accumulated as t += EPS (src/Apps/wilsonflow.cpp:126).
 *          Optionally writes the final links in the .bin layout.
 *   deriv  CONF Nx Ny Nz Nt OUT.bin   computeDerivative(mu) for mu=0..3,
 *          written per site as 4 x 18 doubles (the .bin layout).
 *   exp    IN.bin N OUT.bin           exp(Q) (e^{iQ}) of N 18-double matrices.
 *   time   CONF Nx Ny Nz Nt EPS NSTEPS   seconds for NSTEPS flow steps without
 *          observables and for one SuperObs::compute; one JSON line.
 */
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Actions/puregauge.h"
#include "InputOutput/inputconf.h"
#include "Math/latticemath.h"
#include "Observables/superobs.h"
#include "ParallelTools/parallel.h"

namespace {

void rk3_step(PureGauge& act, GluonField& U, GluonField& Z, double eps) {
    for (int mu = 0; mu < 4; mu++) Z[mu] = act.computeDerivative(mu);
    for (int mu = 0; mu < 4; mu++) U[mu] = exp(Z[mu] * eps * (1.0 / 4.0)) * U[mu];
    for (int mu = 0; mu < 4; mu++) Z[mu] = act.computeDerivative(mu) * (8.0 / 9.0) - Z[mu] * (17.0 / 36.0);
    for (int mu = 0; mu < 4; mu++) U[mu] = exp(Z[mu] * eps) * U[mu];
    for (int mu = 0; mu < 4; mu++) Z[mu] = act.computeDerivative(mu) * (3.0 / 4.0) - Z[mu];
    for (int mu = 0; mu < 4; mu++) U[mu] = exp(Z[mu] * eps) * U[mu];
}

void write_field(GluonField& F, const std::array<int, 4>& n, const char* path) {
    FILE* f = std::fopen(path, "wb");
    if (!f) { std::fprintf(stderr, "ref_flow: cannot write %s\n", path); std::exit(2); }
    for (int t = 0; t < n[3]; t++)
        for (int z = 0; z < n[2]; z++)
            for (int y = 0; y < n[1]; y++)
                for (int x = 0; x < n[0]; x++)
                    for (int mu = 0; mu < 4; mu++)
                        std::fwrite(F[mu].at(x, y, z, t).mat.data(), sizeof(double), 18, f);
    std::fclose(f);
}

std::array<int, 4> dims_from(char** a) {
    return {std::atoi(a[0]), std::atoi(a[1]), std::atoi(a[2]), std::atoi(a[3])};
}

void print_obs(int step, double t, SuperObs& obs) {
    std::printf("%d %.17g %.17g %.17g %.17g\n", step, t, obs.plaq, obs.topc, obs.energy);
}

int usage() {
    std::fprintf(stderr,
                 "usage: ref_flow flow CONF Nx Ny Nz Nt EPS NSTEPS EVERY [OUT.bin]\n"
                 "       ref_flow deriv CONF Nx Ny Nz Nt OUT.bin\n"
                 "       ref_flow exp IN.bin N OUT.bin\n"
                 "       ref_flow time CONF Nx Ny Nz Nt EPS NSTEPS\n");
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) return usage();
    std::string mode = argv[1];
    Parallel::initialize();

    if (mode == "exp") {
        if (argc != 5) return usage();
        long n = std::atol(argv[3]);
        std::vector<double> in(18 * n), out(18 * n);
        FILE* f = std::fopen(argv[2], "rb");
        if (!f || std::fread(in.data(), sizeof(double), in.size(), f) != in.size()) return 3;
        std::fclose(f);
        for (long i = 0; i < n; i++) {
            SU3 q;
            std::memcpy(q.mat.data(), &in[18 * i], 18 * sizeof(double));
            SU3 r = exp(q);
            std::memcpy(&out[18 * i], r.mat.data(), 18 * sizeof(double));
        }
        f = std::fopen(argv[4], "wb");
        std::fwrite(out.data(), sizeof(double), out.size(), f);
        std::fclose(f);
        return 0;
    }

    if ((mode == "flow" && (argc == 10 || argc == 11)) || (mode == "deriv" && argc == 8) ||
        (mode == "time" && argc == 9)) {
        std::array<int, 4> n = dims_from(argv + 3);
        Parallel::createGeometry(n, n);
        GluonField U(n), Z(n);
        LatticeIO::InputConf::readConf(U, argv[2]);
        PureGauge act(6.0);
        act.initAction(&U);
        SuperObs obs;
        obs.initObservable(&U);

        if (mode == "deriv") {
            for (int mu = 0; mu < 4; mu++) Z[mu] = act.computeDerivative(mu);
            write_field(Z, n, argv[7]);
            return 0;
        }

        double eps = std::atof(argv[7]);
        int nsteps = std::atoi(argv[8]);
        if (mode == "time") {
            using clk = std::chrono::steady_clock;
            auto t0 = clk::now();
            for (int s = 0; s < nsteps; s++) rk3_step(act, U, Z, eps);
            auto t1 = clk::now();
            obs.compute();
            auto t2 = clk::now();
            double fs = std::chrono::duration<double>(t1 - t0).count();
            double os = std::chrono::duration<double>(t2 - t1).count();
            double links = 4.0 * n[0] * n[1] * n[2] * n[3];
            std::printf("{\"flow_seconds\": %.6f, \"steps\": %d, \"obs_seconds\": %.6f, "
                        "\"link_updates_per_s\": %.6g, \"plaq\": %.17g}\n",
                        fs, nsteps, os, links * nsteps / fs, obs.plaq);
            return 0;
        }

        int every = std::atoi(argv[9]);
        double t = 0.0;
        obs.compute();
        print_obs(0, t, obs);
        for (int s = 1; s <= nsteps; s++) {
            rk3_step(act, U, Z, eps);
            t += eps;
            if (every > 0 && (s % every == 0 || s == nsteps)) {
                obs.compute();
                print_obs(s, t, obs);
            }
        }
        if (argc == 11) write_field(U, n, argv[10]);
        return 0;
    }
    return usage();
}
