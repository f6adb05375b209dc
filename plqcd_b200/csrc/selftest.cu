// selftest.cu -- known-answer self-test shipped with the library.
//
// The reference's tests/test_comms.c:167-497 applies a gauge-free,
// gamma-free neighbour sum to a point source and prints the result for
// inspection: the output must be non-zero at exactly the 8 neighbours. This
// self-test runs the full operator on the device with unit links:
//   H delta_{y, s, c} has, at the site whose +mu neighbour is y, spin column
//   s of (1 - g_mu) in colour c, and at the site whose -mu neighbour is y,
//   column s of (1 + g_mu); every other site is zero
// with the gamma matrices implied by lib/dirac.c:95-114 / 163-195 /
// 269-311 / 371-398. It then checks gamma5-hermiticity
//   <phi_e, H_eo psi_o> = <g5 H_oe g5 phi_e, psi_o>
// on random SU(3) links and Gaussian spinors, in FP64.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace plqcd;
using cd = std::complex<double>;

namespace {

// (1 - g_mu) columns; (1 + g_mu) = 2 - (1 - g_mu). Row-major 4x4.
void one_minus_gamma(int mu, cd m[16]) {
    const cd I(0, 1);
    cd g[4][16] = {
        {0, 0, -1, 0, 0, 0, 0, -1, -1, 0, 0, 0, 0, -1, 0, 0},
        {0, 0, 0, -I, 0, 0, -I, 0, 0, I, 0, 0, I, 0, 0, 0},
        {0, 0, 0, -1, 0, 0, 1, 0, 0, 1, 0, 0, -1, 0, 0, 0},
        {0, 0, -I, 0, 0, 0, 0, I, I, 0, 0, 0, 0, -I, 0, 0},
    };
    for (int k = 0; k < 16; k++) m[k] = ((k % 5) == 0 ? 1.0 : 0.0) - g[mu][k];
}

struct Dev {
    void *p = nullptr;
    explicit Dev(size_t n) {
        if (cudaMalloc(&p, n) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
    }
    ~Dev() {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int plqcd_selftest(int device, int verbose) {
    clear_error();
    const int L[4] = {4, 4, 4, 6};
    plqcd_lattice *lat = nullptr;
    PLQCD_TRY(plqcd_lattice_create(L, device, nullptr, &lat));
    int rc = PLQCD_OK;
    plqcd_gauge *g = nullptr;
    const long Vh = lat->geom.Vh, V = 2 * Vh;
    const size_t fb = spinor_parity_bytes(Vh, PLQCD_F64);
    Dev aos(sizeof(spinor) * V), fin(fb), fout(fb), fe(fb), fo(fb), t1(fb), t2(fb);
    std::vector<cd> host(12 * V);
    do {
        if (!aos.p || !fin.p || !fout.p || !fe.p || !fo.p || !t1.p || !t2.p) {
            rc = set_error(PLQCD_ERR_NOMEM, "selftest: device allocation");
            break;
        }
        if ((rc = plqcd_gauge_create(lat, PLQCD_F64, 18, &g))) break;
        if ((rc = plqcd_gauge_unit(g))) break;
        // point source on odd half-site h0, spin s, colour c
        const long h0 = 7;
        const int s = 2, c = 1;
        std::vector<cd> src(12 * V, 0.0);
        src[12 * (Vh + h0) + 3 * s + c] = 1.0;
        cudaMemcpy(aos.p, src.data(), sizeof(cd) * src.size(), cudaMemcpyHostToDevice);
        if ((rc = plqcd_spinor_import(lat, (const spinor *)aos.p, PLQCD_ODD, fin.p, PLQCD_F64))) break;
        if ((rc = plqcd_dslash(lat, g, fout.p, fin.p, PLQCD_EVEN, PLQCD_F64, 0))) break;
        cudaMemset(aos.p, 0, sizeof(spinor) * V);
        if ((rc = plqcd_spinor_export(lat, fout.p, PLQCD_F64, PLQCD_EVEN, (spinor *)aos.p))) break;
        cudaMemcpy(host.data(), aos.p, sizeof(cd) * host.size(), cudaMemcpyDeviceToHost);
        // expected result from the site coordinates
        const int L0 = L[0], L1 = L[1], L2 = L[2], L3 = L[3];
        auto coords = [&](long h, int par, int x[4]) {
            long r = h / (L0 / 2);
            x[1] = r % L1;
            x[2] = (r / L1) % L2;
            x[3] = (int)(r / L1 / L2);
            x[0] = 2 * (h % (L0 / 2)) + ((x[1] + x[2] + x[3] + par) & 1);
        };
        int y[4];
        coords(h0, 1, y);
        double err = 0;
        int nonzero = 0;
        for (long h = 0; h < Vh; h++) {
            int x[4];
            coords(h, 0, x);
            cd want[12] = {};
            for (int mu = 0; mu < 4; mu++) {
                cd m[16];
                one_minus_gamma(mu, m);
                int xp[4] = {x[0], x[1], x[2], x[3]}, xm[4] = {x[0], x[1], x[2], x[3]};
                xp[mu] = (x[mu] + 1) % L[mu];
                xm[mu] = (x[mu] + L[mu] - 1) % L[mu];
                if (!memcmp(xp, y, sizeof xp))
                    for (int sp = 0; sp < 4; sp++) want[3 * sp + c] += m[4 * sp + s];
                if (!memcmp(xm, y, sizeof xm))
                    for (int sp = 0; sp < 4; sp++) want[3 * sp + c] += ((sp == s) ? 2.0 : 0.0) - m[4 * sp + s];
            }
            bool any = false;
            for (int k = 0; k < 12; k++) {
                err = std::max(err, std::abs(host[12 * h + k] - want[k]));
                if (std::abs(host[12 * h + k]) > 0) any = true;
            }
            nonzero += any;
        }
        if (verbose) fprintf(stderr, "plqcd selftest: point source, %d non-zero sites, max error %.3e\n", nonzero, err);
        if (err != 0.0 || nonzero != 8) {
            rc = set_error(PLQCD_ERR_STATE, "selftest: point-source check failed (%d sites, error %.3e)", nonzero, err);
            break;
        }
        // gamma5-hermiticity on random fields
        if ((rc = plqcd_gauge_random(g, 99))) break;
        if ((rc = plqcd_spinor_gaussian(lat, fe.p, PLQCD_F64, PLQCD_EVEN, 1))) break;
        if ((rc = plqcd_spinor_gaussian(lat, fo.p, PLQCD_F64, PLQCD_ODD, 2))) break;
        if ((rc = plqcd_dslash(lat, g, t1.p, fo.p, PLQCD_EVEN, PLQCD_F64, 0))) break;
        if ((rc = plqcd_dslash(lat, g, t2.p, fe.p, PLQCD_ODD, PLQCD_F64, PLQCD_DSLASH_G5_IN | PLQCD_DSLASH_G5_OUT)))
            break;
        std::vector<cd> a(12 * Vh), b(12 * Vh), pe(12 * Vh), po(12 * Vh);
        auto fetch = [&](void *f, int par, std::vector<cd> &dst) {
            plqcd_spinor_export(lat, f, PLQCD_F64, par, (spinor *)aos.p);
            cudaDeviceSynchronize();
            cudaMemcpy(dst.data(), (char *)aos.p + par * Vh * sizeof(spinor), sizeof(spinor) * Vh,
                       cudaMemcpyDeviceToHost);
        };
        fetch(t1.p, 0, a);
        fetch(t2.p, 1, b);
        fetch(fe.p, 0, pe);
        fetch(fo.p, 1, po);
        cd lhs = 0, rhs = 0;
        for (long k = 0; k < 12 * Vh; k++) {
            lhs += std::conj(pe[k]) * a[k];
            rhs += std::conj(b[k]) * po[k];
        }
        const double herm = std::abs(lhs - rhs) / std::abs(lhs);
        if (verbose) fprintf(stderr, "plqcd selftest: gamma5-hermiticity relative deviation %.3e\n", herm);
        if (!(herm < 1e-12)) {
            rc = set_error(PLQCD_ERR_STATE, "selftest: gamma5-hermiticity violated (%.3e)", herm);
            break;
        }
    } while (0);
    if (cudaGetLastError() != cudaSuccess && rc == PLQCD_OK) rc = set_error(PLQCD_ERR_CUDA, "selftest: CUDA error");
    if (g) plqcd_gauge_destroy(g);
    plqcd_lattice_destroy(lat);
    return rc;
}
