// alphabet.cuh - the texts' alphabet and the packed code stream the ranking keys and the merge
// records are cut from.
//
// Every byte value present in the texts gets a code, in byte order (so code order is byte order),
// of b = bit_width(sigma - 1) bits (at least 1). The codes of the concatenation are packed into a
// big-endian bit stream of 64-bit words: character q occupies bits [q*b, (q+1)*b) counted from the
// most significant bit of word 0, so 64 bits taken at bit q*b hold characters q, q+1, ... with
// character q on top and compare as integers exactly as the byte strings compare. Positions past a
// text's end read code 0 (the smallest character): a shorter suffix can tie with a longer one there
// but never sort after it, and the length tags and text ends separate them (as zero padding does
// for bytes). DNA packs 29 characters into a ranking key (bytes: 7) and 64 into a merge record's 16
// bytes (bytes: 16).
#pragma once

#include "common.cuh"

namespace sadcs {

struct CodeTable {
    uint8_t code[256];
};

// counts[c] += occurrences of byte c inside the texts (zeroed by the caller). Sixteen bytes per
// thread and iteration (one 16-byte load; the text buffer is 16-byte aligned and padded), counted
// in one shared histogram per warp so that only lanes of one warp contend for a counter.
__global__ void __launch_bounds__(256) alphabetHistogram(const uint8_t* __restrict__ text, uint32_t total,
                                                         TextSet texts, uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    uint32_t* mine = h[threadIdx.x >> 5];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x * 16;
    for (uint64_t base = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 16; base < total;
         base += stride) {
        const uint4 v = *reinterpret_cast<const uint4*>(text + base);
        const uint32_t words[4] = {v.x, v.y, v.z, v.w};
        if (texts.count <= 1 && base + 16 <= total) {  // one text, all 16 bytes inside it
#pragma unroll
            for (int b = 0; b < 16; b++) atomicAdd(&mine[(words[b >> 2] >> (8 * (b & 3))) & 0xFF], 1u);
        } else {
            // 16 bytes at a multiple of 16 lie in one 32-byte block, hence in one text's range
            const uint64_t end = min(static_cast<uint64_t>(total), static_cast<uint64_t>(texts.endOf(static_cast<uint32_t>(base))));
#pragma unroll
            for (int b = 0; b < 16; b++) {
                if (base + b < end) atomicAdd(&mine[(words[b >> 2] >> (8 * (b & 3))) & 0xFF], 1u);
            }
        }
    }
    __syncthreads();
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) sum += h[w][threadIdx.x];
    if (sum) atomicAdd(counts + threadIdx.x, sum);
}

// The code stream in groups: a group of G = 64 / gcd(bits, 64) characters fills exactly
// G * bits / 64 whole words (DNA: 32 characters, one word; 6-bit codes: 32 characters, three words),
// so one thread packs a group from its bytes read by 16-byte loads (8-byte for 8-bit codes) and
// writes its words. Positions past the end of the concatenation read code 0. The byte-to-code table
// is copied to shared memory first: indexed by data, a kernel-parameter table would serialise a
// warp's lookups.
__host__ __device__ constexpr uint32_t packGroupChars(uint32_t bits) {
    return 64u / (bits & (0u - bits));  // gcd(bits, 64): the lowest set bit of bits (bits <= 8)
}

__global__ void __launch_bounds__(256) packCodes(const uint8_t* __restrict__ text, uint32_t total, CodeTable table,
                                                 uint32_t bits, uint64_t words, uint64_t* __restrict__ packed) {
    __shared__ uint8_t code[256];
    code[threadIdx.x] = table.code[threadIdx.x];
    __syncthreads();
    const uint32_t G = packGroupChars(bits), perGroup = G * bits / 64;
    const uint64_t group = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t firstWord = group * perGroup;
    if (firstWord >= words) return;
    const uint64_t firstChar = group * G;
    uint64_t acc = 0, out = firstWord;
    uint32_t filled = 0;
    auto put = [&](uint32_t c) {
        if (filled + bits <= 64) {
            acc = (acc << bits) | c;
            filled += bits;
            if (filled == 64) {
                if (out < words) packed[out] = acc;
                out++;
                acc = 0;
                filled = 0;
            }
        } else {  // the character straddles two words
            const uint32_t over = filled + bits - 64;
            if (out < words) packed[out] = (acc << (bits - over)) | (c >> over);
            out++;
            acc = c & ((1u << over) - 1);
            filled = over;
        }
    };
    const uint32_t step = G >= 16 ? 16 : 8;
    for (uint32_t piece = 0; piece < G; piece += step) {
        const uint64_t q0 = firstChar + piece;
        uint8_t bytes[16];
        if (q0 + step <= total) {  // inside the text: one aligned vector load
            if (step == 16) {
                *reinterpret_cast<uint4*>(bytes) = *reinterpret_cast<const uint4*>(text + q0);
            } else {
                *reinterpret_cast<uint2*>(bytes) = *reinterpret_cast<const uint2*>(text + q0);
            }
        } else {
            for (uint32_t k = 0; k < step; k++) bytes[k] = q0 + k < total ? text[q0 + k] : 0;
        }
        for (uint32_t k = 0; k < step; k++) put(q0 + k < total ? code[bytes[k]] : 0u);
    }
}

// 64 bits of the code stream starting at stream bit `bit`.
__device__ __forceinline__ uint64_t streamBits(const uint64_t* __restrict__ packed, uint64_t bit) {
    const uint64_t w = bit >> 6;
    const uint32_t o = static_cast<uint32_t>(bit & 63);
    const uint64_t hi = __ldg(packed + w);
    return o ? (hi << o) | (__ldg(packed + w + 1) >> (64 - o)) : hi;
}

// The code of character q.
__device__ __forceinline__ uint32_t charCode(const TextSet& texts, uint64_t q) {
    return static_cast<uint32_t>(streamBits(texts.packed, q * texts.bits) >> (64 - texts.bits));
}

// The byte of character q.
__device__ __forceinline__ uint8_t charByte(const TextSet& texts, uint64_t q) {
    return __ldg(texts.decode + charCode(texts, q));
}

// Bits per character and characters per ranking key for an alphabet of sigma symbols.
struct KeyShape {
    uint32_t bits;      // per character
    uint32_t chars;     // characters per 64-bit ranking key
    uint32_t tagBits;   // length tag below them
    uint32_t record;    // characters in a merge record's 128 bits
};

inline KeyShape keyShape(uint32_t sigma) {
    KeyShape k{};
    uint32_t b = 1;
    while (b < 8 && (1u << b) < sigma) b++;
    k.bits = b;
    uint32_t c = 64 / b;
    auto width = [](uint32_t x) {
        uint32_t w = 0;
        while (x) {
            w++;
            x >>= 1;
        }
        return w;
    };
    while (c * b + width(c) > 64) c--;
    k.chars = c;
    k.tagBits = width(c);
    k.record = 128 / b;
    return k;
}

// Number of stream words for a concatenation of `span` bytes, with room for 64-bit reads at any
// position up to span + 64.
inline uint64_t packedWords(uint64_t span, uint32_t bits) {
    return ((span + 160) * bits + 63) / 64 + 4;
}

}  // namespace sadcs
