/*
 * mdx_oracle.c -- CPU oracle for the stable m-way partition (m-discriminator).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker against which the CUDA
 * path is compared; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product (mdiscriminator_b200/libmdx.so) never
 * links, loads or calls it.
 *
 * It is a plain-C restatement of the reference's sequential implementation:
 *
 *   seqMdiscr<DISCR,MEASURE>      cuda_code/SeqMdiscr.h:10-57
 *     pass 1  count classes                       SeqMdiscr.h:29-32
 *     offsets exclusive scan of the counts        SeqMdiscr.h:34-38
 *     pass 2  scatter with per-class cursors,
 *             zero the head-flag array            SeqMdiscr.h:40-45
 *     sizes[offset_c] = count_c for every c       SeqMdiscr.h:47-49
 *
 *   tupleToSizeArray (tuple -> head flags)        cuda_code/HelpersCommon.h:296-311
 *   validate of mdiscrSegm: seqMdiscr per segment cuda_code/MdiscrSegmTest.cu:8-41
 *   record elements (ModArray<N,2>, key = x[0])   cuda_code/MdiscrHost_arrays.cu.h:26-36,44-96
 *
 * Discriminators (cuda_code/HelpersCommon.h):
 *   MOD  : class = key % m   (Mod<N>  :1200-1210)
 *   MASK : class = key & (m-1), m a power of two  (Mod4 :587-596, Mod8 :840-849)
 *
 * Head-flag sizes: the reference writes sizes[offset_c] = count_c for every
 * class in increasing c.  An empty class therefore writes 0 at the offset of
 * the next class (which overwrites it) or, for trailing empty classes, one
 * slot past the end of the array.  Inside [0, n) this equals "count_c at
 * offset_c for every non-empty class, 0 elsewhere", which is what the oracle
 * writes; the one-past-end write is not reproduced (it is out of bounds).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MDX_ORACLE_MAX_M 65536u

enum { ORACLE_DISCR_MOD = 0, ORACLE_DISCR_MASK = 1 };

static inline uint32_t oracle_class(uint32_t key, int kind, uint32_t m) {
    return kind == ORACLE_DISCR_MASK ? (key & (m - 1u)) : (key % m);
}

/* Generic stable partition over elements of `width` bytes whose class key is
 * the first 32-bit word of the element (little-endian record {key, payload}).
 * Returns 0 on success, -1 on bad arguments. */
static int oracle_partition_bytes(uint64_t n, const void* in_v, void* out_v, size_t width,
                                  int kind, uint32_t m, uint32_t* sizes_tuple,
                                  uint32_t* headflags) {
    const unsigned char* in = (const unsigned char*)in_v;
    unsigned char* out = (unsigned char*)out_v;
    if (m == 0 || m > MDX_ORACLE_MAX_M) return -1;
    if (kind == ORACLE_DISCR_MASK && (m & (m - 1u)) != 0) return -1;
    uint64_t* count = (uint64_t*)calloc(m, sizeof(uint64_t));
    uint64_t* cursor = (uint64_t*)calloc(m, sizeof(uint64_t));
    if (!count || !cursor) { free(count); free(cursor); return -1; }

    /* pass 1: reduction[eq_class]++ (SeqMdiscr.h:29-32) */
    for (uint64_t i = 0; i < n; i++) {
        uint32_t key;
        memcpy(&key, in + i * width, sizeof(key));
        count[oracle_class(key, kind, m)]++;
    }
    /* offsets = exclusive scan (SeqMdiscr.h:34-38) */
    uint64_t acc = 0;
    for (uint32_t c = 0; c < m; c++) { cursor[c] = acc; acc += count[c]; }
    /* pass 2: out[count[c]++ + offsets[c]] = in[i] (SeqMdiscr.h:40-45) */
    if (headflags) memset(headflags, 0, (size_t)n * sizeof(uint32_t));
    for (uint64_t i = 0; i < n; i++) {
        uint32_t key;
        memcpy(&key, in + i * width, sizeof(key));
        uint32_t c = oracle_class(key, kind, m);
        memcpy(out + (cursor[c]++) * width, in + i * width, width);
    }
    /* head-flag sizes (SeqMdiscr.h:47-49), restricted to [0, n) */
    if (headflags) {
        acc = 0;
        for (uint32_t c = 0; c < m; c++) {
            if (count[c] > 0) headflags[acc] = (uint32_t)count[c];
            acc += count[c];
        }
    }
    if (sizes_tuple)
        for (uint32_t c = 0; c < m; c++) sizes_tuple[c] = (uint32_t)count[c];
    free(count);
    free(cursor);
    return 0;
}

/* Stable partition of n u32 values.  sizes_tuple: m counts (may be NULL);
 * headflags: n entries in the reference's head-flag form (may be NULL). */
int mdx_oracle_partition_u32(uint64_t n, const uint32_t* in, uint32_t* out, int kind,
                             uint32_t m, uint32_t* sizes_tuple, uint32_t* headflags) {
    return oracle_partition_bytes(n, in, out, 4, kind, m, sizes_tuple, headflags);
}

/* Stable partition of n 8-byte records {u32 key, u32 payload}; class from key. */
int mdx_oracle_partition_rec8(uint64_t n, const uint64_t* in, uint64_t* out, int kind,
                              uint32_t m, uint32_t* sizes_tuple, uint32_t* headflags) {
    return oracle_partition_bytes(n, in, out, 8, kind, m, sizes_tuple, headflags);
}

/* Segmented stable partition: every segment [offsets[s], offsets[s+1]) is
 * partitioned independently (MdiscrSegmTest.cu:21-38 validates exactly this).
 * seg_sizes: S*m counts, row s = class sizes of segment s (may be NULL).
 * headflags: n entries, head-flag sizes relative to each segment start, the
 * form mdiscrSegm writes into new_sizes (MdiscrSegmKernels.cu:89-114). */
int mdx_oracle_partition_segmented(uint64_t n, const void* in, void* out, size_t width,
                                   const uint64_t* offsets, uint64_t num_segments,
                                   int kind, uint32_t m, uint32_t* seg_sizes,
                                   uint32_t* headflags) {
    if (width != 4 && width != 8) return -1;
    if (num_segments > 0 && (offsets[0] != 0 || offsets[num_segments] != n)) return -1;
    for (uint64_t s = 0; s < num_segments; s++) {
        uint64_t a = offsets[s], b = offsets[s + 1];
        if (b < a) return -1;
        int rc = oracle_partition_bytes(b - a, (const unsigned char*)in + a * width,
                                        (unsigned char*)out + a * width, width, kind, m,
                                        seg_sizes ? seg_sizes + s * m : NULL,
                                        headflags ? headflags + a : NULL);
        if (rc) return rc;
    }
    return 0;
}

/* Head-flag segment sizes -> segment offsets.  flags[i] = length of the
 * segment starting at i, 0 elsewhere (populateSizesArray,
 * HelpersCommon.h:105-151).  Writes at most max_segments+1 offsets and
 * returns the number of segments, or -1 if the flags are malformed (a segment
 * running past n, or a non-zero flag inside a segment). */
int64_t mdx_oracle_flags_to_offsets(uint64_t n, const int32_t* flags, uint64_t* offsets,
                                    uint64_t max_segments) {
    uint64_t s = 0, i = 0;
    while (i < n) {
        int32_t len = flags[i];
        if (len <= 0 || i + (uint64_t)len > n) return -1;
        for (uint64_t j = i + 1; j < i + (uint64_t)len; j++)
            if (flags[j] != 0) return -1;
        if (s >= max_segments) return -1;
        offsets[s++] = i;
        i += (uint64_t)len;
    }
    offsets[s] = n;
    return (int64_t)s;
}

/* tupleToSizeArray (HelpersCommon.h:296-311): sizes tuple -> head flags. */
void mdx_oracle_tuple_to_headflags(uint64_t n, const uint32_t* sizes, uint32_t m,
                                   uint32_t* headflags) {
    memset(headflags, 0, (size_t)n * sizeof(uint32_t));
    uint64_t off = 0;
    for (uint32_t c = 0; c < m && off < n; c++) {
        if (sizes[c] > 0) headflags[off] = sizes[c];
        off += sizes[c];
    }
}

/* splitmix64: the seeded generator every test and the bench use for inputs. */
static inline uint64_t splitmix64_next(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Uniform u32 values in [0, 2^31) from splitmix64(seed). */
void mdx_oracle_fill_uniform_u32(uint64_t n, uint64_t seed, uint32_t* out) {
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; i++) out[i] = (uint32_t)(splitmix64_next(&s) >> 33);
}
