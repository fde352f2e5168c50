/* Test infrastructure: drives every entry point of the oracle (ymoracle.c) on
 * small, odd and degenerate lattices under AddressSanitizer and
 * UndefinedBehaviorSanitizer (`make -C oracle sanitize`).  Any out-of-bounds
 * neighbour index, overflow or use of uninitialised allocation aborts the run
 * with the sanitizer's report; a clean run prints "sanitize ok". */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ymoracle.h"

static int check_lattice(const int n[4]) {
    const long V = (long)n[0] * n[1] * n[2] * n[3];
    const long links = 4 * V;
    double* U = malloc(sizeof(double) * 18 * links);
    double* Z = malloc(sizeof(double) * 18 * links);
    double* Zmu = malloc(sizeof(double) * 18 * V);
    double table[5 * 8];
    double obs[3], uni[2];
    if (!U || !Z || !Zmu) return 1;
    yo_gen_cold(U, n);
    yo_superobs(U, n, obs);
    if (fabs(obs[0] - 1.0) > 1e-14) return 2;
    yo_gen_expiah(U, n, 0.35, 5, 1);
    yo_gen_haar_mix(U, n, 0.2, 5, 1);
    for (int mu = 0; mu < 4; mu++) yo_derivative(U, n, mu, Zmu);
    yo_flow_step(U, Z, n, 0.01);
    if (yo_flow(U, n, 0.01, 3, 1, table) != 4) return 3;
    yo_superobs(U, n, obs);
    yo_reunitarize(U, links);
    yo_unitarity(U, links, uni);
    if (!(uni[0] < 1e-12) || !isfinite(obs[1])) return 4;
    int even = 1;
    for (int i = 0; i < 4; i++) even = even && n[i] % 2 == 0;
    if (even) {
        yo_gen_cold(U, n);
        yo_gen_metropolis_cb(U, n, 6.0, 0.24, 1, 2, 9, 0);
        yo_gen_metropolis(U, n, 6.0, 0.24, 1, 2, 9);
    }
    free(U);
    free(Z);
    free(Zmu);
    return 0;
}

int main(void) {
    const int lattices[][4] = {{1, 1, 1, 1}, {1, 2, 3, 4}, {2, 2, 2, 2}, {3, 4, 5, 6}, {5, 1, 2, 3}, {4, 4, 4, 4}};
    for (size_t i = 0; i < sizeof(lattices) / sizeof(lattices[0]); i++) {
        const int r = check_lattice(lattices[i]);
        if (r) {
            printf("lattice %zu failed check %d\n", i, r);
            return 1;
        }
    }
    double q[18] = {0}, e[18];
    q[0] = 0.3;
    q[8] = -0.1;
    q[16] = -0.2;
    yo_exp(q, e);
    printf("sanitize ok\n");
    return 0;
}
