/*
 * murmur_golden.cpp -- TEST INFRASTRUCTURE ONLY.
 * Prints golden Murmur2 values computed by the reference's own software
 * hash functions (unit_tests/bloom_and_hash/sw_murmur2/murmur2.cpp, linked
 * from its source with its main() renamed) as JSON lines: key, seed,
 * MurmurHash2(key, 4, seed), MurmurHash2_KeyLen4(key, seed).
 */
#include <cstdint>
#include <cstdio>
uint32_t MurmurHash2(const void *key, int len, uint32_t seed);
uint32_t MurmurHash2_KeyLen4(const void *key, uint32_t seed);
int main()
{
    uint32_t keys[64];
    int nk = 0;
    for (uint32_t k = 0; k < 32; k++) keys[nk++] = k;
    const uint32_t extra[] = {100u, 1000u, 65535u, 65536u, 99999u, 100000u, 999999u, 1000000u,
                              9999999u, 0x7fffffffu, 0x80000000u, 0xffffffffu, 123456789u, 2718281u,
                              31415926u, 4096u};
    for (uint32_t e : extra) keys[nk++] = e;
    std::printf("[\n");
    bool first = true;
    for (uint32_t seed = 0; seed < 5; seed++)
        for (int i = 0; i < nk; i++) {
            uint32_t k = keys[i];
            std::printf("%s{\"key\": %u, \"seed\": %u, \"murmur2\": %u, \"keylen4\": %u}", first ? "" : ",\n", k,
                        seed, MurmurHash2(&k, 4, seed), MurmurHash2_KeyLen4(&k, seed));
            first = false;
        }
    std::printf("\n]\n");
    return 0;
}
