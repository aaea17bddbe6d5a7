/*
 * Oracle (test infrastructure only): Philox4x32-10, the uniform and normal
 * draws, and key derivation, restated from the reference:
 *   src/backends/cpu/kernels/philox.inl:15-110 (round, counter and key words)
 *   src/backends/cpu/kernels/standard_normal.inl:19-50 (uniform_open_closed,
 *     Box-Muller pair, cosine branch for even counters)
 *   src/backends/cpu/kernels/random_key.inl:13 (derive_key)
 * The Philox multipliers and Weyl constants are the published Random123
 * constants (Salmon et al., SC'11).
 */
#include "oracle.h"

#include <math.h>

enum { DOMAIN_DRAW = 0, DOMAIN_KEY_DERIVATION = 1 };

static void philox_round(uint32_t c[4], const uint32_t k[2])
{
	const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
	const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
	const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
	const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
	const uint32_t n0 = hi1 ^ c[1] ^ k[0];
	const uint32_t n2 = hi0 ^ c[3] ^ k[1];
	c[0] = n0;
	c[1] = lo1;
	c[2] = n2;
	c[3] = lo0;
}

void oracle_philox4x32_10(const uint32_t counter[4], const uint32_t key[2], uint32_t out[4])
{
	uint32_t c[4] = { counter[0], counter[1], counter[2], counter[3] };
	uint32_t k[2] = { key[0], key[1] };
	philox_round(c, k);
	for (int round = 1; round < 10; ++round)
	{
		k[0] += 0x9E3779B9u;
		k[1] += 0xBB67AE85u;
		philox_round(c, k);
	}
	for (int i = 0; i < 4; ++i)
		out[i] = c[i];
}

double oracle_uniform_open_closed(uint64_t bits)
{
	return (double)((bits >> 11) + 1) * (1.0 / 9007199254740992.0);
}

static void block_halves(uint64_t key, uint64_t block, uint32_t domain, uint64_t halves[2])
{
	const uint32_t counter[4] = { (uint32_t)block, (uint32_t)(block >> 32), 0u, domain };
	const uint32_t k[2] = { (uint32_t)key, (uint32_t)(key >> 32) };
	uint32_t out[4];
	oracle_philox4x32_10(counter, k, out);
	halves[0] = ((uint64_t)out[1] << 32) | out[0];
	halves[1] = ((uint64_t)out[3] << 32) | out[2];
}

void oracle_standard_normal_pair(uint64_t key, uint64_t block, double out[2])
{
	uint64_t halves[2];
	block_halves(key, block, DOMAIN_DRAW, halves);
	const double radius = sqrt(-2.0 * log(oracle_uniform_open_closed(halves[0])));
	const double angle = 6.283185307179586476925 * oracle_uniform_open_closed(halves[1]);
	out[0] = radius * cos(angle);
	out[1] = radius * sin(angle);
}

uint64_t oracle_derive_key(uint64_t key, uint64_t data)
{
	uint64_t halves[2];
	block_halves(key, data, DOMAIN_KEY_DERIVATION, halves);
	return halves[0];
}
