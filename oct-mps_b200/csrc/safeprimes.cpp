// Multiplier table for the multiply-with-carry (MWC) generators.
//
// The reference seeds one MWC generator per lane and per stream from the
// first column of `safeprimes_base32.txt` (src/octmps_kernel.cuh:74-76,
// 95-105), a file that is not shipped with it.  A valid MWC multiplier `a`
// for base b = 2^32 makes p = a*2^32 - 1 and (p - 1)/2 = a*2^31 - 1 both
// prime, which gives the generator its full period (p - 1)/2.  This file
// regenerates such a list deterministically: every a < 2^32 that passes,
// scanned downward from 2^32 - 1.  Primality is the deterministic
// Miller-Rabin test for 64-bit integers with the seven bases found by
// J. Sinclair (2, 325, 9375, 28178, 450775, 9780504, 1795265022), after a
// sieve by the odd primes below 2^16.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "octmps_host.h"

namespace {

typedef unsigned __int128 u128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) {
    return (uint64_t)((u128)a * b % m);
}

uint64_t powmod(uint64_t a, uint64_t e, uint64_t m) {
    uint64_t r = 1;
    a %= m;
    while (e) {
        if (e & 1) r = mulmod(r, a, m);
        a = mulmod(a, a, m);
        e >>= 1;
    }
    return r;
}

// Strong probable-prime test of odd n > 2 to base a.
bool sprp(uint64_t n, uint64_t a) {
    a %= n;
    if (a == 0) return true;
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; ++s; }
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) return true;
    for (int i = 1; i < s; ++i) {
        x = mulmod(x, x, n);
        if (x == n - 1) return true;
        if (x == 1) return false;
    }
    return false;
}

bool is_prime_u64(uint64_t n) {
    static const uint64_t bases[7] = {2ull, 325ull, 9375ull, 28178ull,
                                      450775ull, 9780504ull, 1795265022ull};
    if (n < 2) return false;
    if ((n & 1) == 0) return n == 2;
    for (uint64_t a : bases)
        if (!sprp(n, a)) return false;
    return true;
}

struct SmallPrime {
    uint32_t r;      // the prime
    uint32_t inv32;  // 2^-32 mod r: a == inv32 makes a*2^32 - 1 divisible by r
    uint32_t inv31;  // 2^-31 mod r: a == inv31 makes a*2^31 - 1 divisible by r
};

std::vector<SmallPrime> small_primes() {
    const uint32_t limit = 1u << 16;
    std::vector<char> comp(limit, 0);
    std::vector<SmallPrime> out;
    for (uint32_t i = 3; i < limit; i += 2) {
        if (comp[i]) continue;
        for (uint64_t j = (uint64_t)i * i; j < limit; j += 2ull * i) comp[j] = 1;
        // inverse of 2^k mod i via Fermat: 2^(k*(i-2)) mod i
        uint64_t inv2 = (i + 1) / 2;  // 2^-1 mod i
        uint32_t inv31 = (uint32_t)powmod(inv2, 31, i);
        uint32_t inv32 = (uint32_t)mulmod(inv31, inv2, i);
        out.push_back({i, inv32, inv31});
    }
    return out;
}

}  // namespace

extern "C" int octmps_safeprimes_generate(uint32_t *out, uint64_t count) {
    if (!out && count) return OCTMPS_ERR_INVALID_ARG;
    if (count == 0) return OCTMPS_OK;
    const std::vector<SmallPrime> sp = small_primes();
    const uint32_t block = 1u << 18;
    uint64_t found = 0;
    uint64_t hi = 0xffffffffull;  // next candidate, scanning downward
    // Blocks are sieved and tested in parallel and appended in order.
    const int par = 16;
    while (found < count && hi >= 0x80000000ull) {
        std::vector<std::vector<uint32_t>> res(par);
        uint64_t his[par];
        for (int b = 0; b < par; ++b) his[b] = hi >= (uint64_t)b * block ? hi - (uint64_t)b * block : 0;
#pragma omp parallel for schedule(dynamic, 1)
        for (int b = 0; b < par; ++b) {
            uint64_t top = his[b];
            if (top < 0x80000000ull) continue;
            uint64_t lo = top + 1 >= block ? top + 1 - block : 0;
            if (lo < 0x80000000ull) lo = 0x80000000ull;
            std::vector<char> bad(top - lo + 1, 0);
            for (const SmallPrime &s : sp) {
                // first a >= lo with a % r == residue
                for (uint32_t resid : {s.inv32, s.inv31}) {
                    uint64_t start = lo + ((resid + s.r - (uint32_t)(lo % s.r)) % s.r);
                    for (uint64_t a = start; a <= top; a += s.r) bad[a - lo] = 1;
                }
            }
            for (uint64_t a = top + 1; a-- > lo;) {
                if (bad[a - lo]) continue;
                uint64_t q = (a << 31) - 1;
                uint64_t p = (a << 32) - 1;
                if (!sprp(q, 2) || !sprp(p, 2)) continue;
                if (is_prime_u64(q) && is_prime_u64(p)) res[b].push_back((uint32_t)a);
            }
        }
        for (int b = 0; b < par && found < count; ++b)
            for (uint32_t a : res[b]) {
                if (found == count) break;
                out[found++] = a;
            }
        hi = hi >= (uint64_t)par * block ? hi - (uint64_t)par * block : 0;
    }
    return found == count ? OCTMPS_OK : OCTMPS_ERR_INVALID_ARG;
}

extern "C" int octmps_safeprimes_write(const char *path, uint64_t count) {
    std::vector<uint32_t> a(count);
    int st = octmps_safeprimes_generate(a.data(), count);
    if (st != OCTMPS_OK) return st;
    FILE *f = fopen(path, "w");
    if (!f) return OCTMPS_ERR_IO;
    // Columns: multiplier a, then the high and low 32-bit words of the
    // safe prime a*2^32 - 1.  The reference reads only the first column.
    for (uint64_t i = 0; i < count; ++i)
        fprintf(f, "%u %u %u\n", a[i], a[i] - 1u, 0xffffffffu);
    fclose(f);
    return OCTMPS_OK;
}
