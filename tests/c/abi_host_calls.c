/* A plain C caller of the C ABI: includes include/afhe.h, links libafhe.so,
 * and makes the host-only calls a reference-side binding makes before it
 * has a device (prime search, roots, Galois elements, parameter checks).
 * Prints one line per check; exits non-zero on the first failure. */
#include <stdio.h>
#include <string.h>

#include "afhe.h"

static uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t m) {
    unsigned __int128 r = 1, x = b % m;
    while (e) {
        if (e & 1) r = r * x % m;
        x = x * x % m;
        e >>= 1;
    }
    return (uint64_t)r;
}

int main(void) {
    const uint32_t log_n = 13;
    const uint64_t two_n = 2ull << log_n;
    uint64_t q[3], p[1];
    if (afhe_find_ntt_primes(log_n, 50, 3, NULL, 0, q) != AFHE_OK) return 1;
    if (afhe_find_ntt_primes(log_n, 60, 1, q, 3, p) != AFHE_OK) return 2;
    for (int i = 0; i < 3; ++i)
        if (q[i] % two_n != 1 || q[i] >= (1ull << 50)) return 3;
    printf("primes ok\n");

    const uint64_t psi = afhe_min_primitive_root(log_n, q[0]);
    if (pow_mod(psi, 1ull << log_n, q[0]) != q[0] - 1) return 4;
    const uint64_t inv = afhe_inv_mod(psi, q[0]);
    if ((unsigned __int128)inv * psi % q[0] != 1) return 5;
    printf("root ok\n");

    if (afhe_galois_elt(log_n, 1) != 5 || afhe_galois_elt(log_n, 0) != 1) return 6;
    if (pow_mod(5, 1, two_n) * afhe_galois_elt(log_n, -1) % two_n != 1) return 7;
    printf("galois ok\n");

    afhe_params prm;
    memset(&prm, 0, sizeof prm);
    prm.log_n = 9;  /* below the supported range */
    prm.num_q = 3;
    prm.num_p = 1;
    prm.alpha = 1;
    memcpy(prm.q, q, sizeof q);
    memcpy(prm.p, p, sizeof p);
    prm.poly_words = prm.key_words = 1u << 16;
    afhe_ctx* ctx = NULL;
    if (afhe_ctx_create(&prm, &ctx) != AFHE_E_ARG || ctx != NULL) return 8;
    if (strlen(afhe_last_error()) == 0) return 9;
    prm.log_n = log_n;
    prm.psi_q[0] = 1;  /* not a primitive root */
    if (afhe_ctx_create(&prm, &ctx) != AFHE_E_ARG || ctx != NULL) return 10;
    if (afhe_sync(NULL) != AFHE_E_ARG) return 11;
    printf("checks ok: %s\n", afhe_status_string(AFHE_E_ARG));
    return 0;
}
