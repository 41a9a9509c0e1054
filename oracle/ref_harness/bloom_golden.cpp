/*
 * bloom_golden.cpp -- TEST INFRASTRUCTURE ONLY.
 * Runs the reference's software Bloom filter (unit_tests/bloom_and_hash/
 * sw_bloom/bloom_murmur2.hpp:90-134: 3 hashes with seeds seed..seed+2,
 * bucket = hash % num_buckets) over a seeded key stream with repeats and
 * prints, per key, whether check_and_insert reported it new (the kernel's
 * "valid" bit).  Output: JSON {bits, seed, keys, valid}.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>  /* the header uses memset without including it */
#include "bloom_murmur2.hpp"
int main(int argc, char **argv)
{
    const int bits = argc > 1 ? std::atoi(argv[1]) : 16;
    const int n = argc > 2 ? std::atoi(argv[2]) : 20000;
    const int seed = 1;
    BloomFilter bf(1 << bits, 3, seed);
    uint64_t s = 0x9e3779b97f4a7c15ull;
    std::printf("{\"bits\": %d, \"seed\": %d, \"keys\": [", bits, seed);
    int *keys = (int *)std::malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        keys[i] = (int)((s >> 33) % 50000u);   /* repeats guaranteed */
        std::printf("%s%d", i ? ", " : "", keys[i]);
    }
    std::printf("], \"valid\": [");
    for (int i = 0; i < n; i++) std::printf("%s%d", i ? ", " : "", bf.check_and_insert(keys[i]) ? 0 : 1);
    std::printf("]}\n");
    std::free(keys);
    return 0;
}
