/*
 * fss_oracle.c — CPU restatement of the FastFss evaluation hot path (TEST INFRASTRUCTURE).
 *
 * This file is the checker for the CUDA library, never part of it: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it. It is a plain-C
 * restatement of the reference's per-element algorithms; each function names the
 * reference file:line it follows (paths relative to the FastFunctionSecretSharing tree).
 *
 * Conventions shared with the reference:
 *   - AES-128 is FIPS-197 byte order (src/impl/aes.h:10-18 loads state words big-endian).
 *   - The PRG keys AES with the 16-byte node seed and encrypts the little-endian uint64
 *     array {0,1,2,...}: block j is (2j, 2j+1) (src/impl/dcf.h:197-198,230-233).
 *   - A node seed has bit 0 of its low word cleared (MASK_MSB63, src/impl/dcf.h:197,205)
 *     and that bit of a fresh child block is its control bit t.
 *   - Ring elements live in uint64_t and are reduced mod 2^(8*elementSize) on store.
 *
 * The host is assumed little-endian (x86-64), as the reference's uint64 views of byte
 * buffers are.
 */
#include "fss_oracle.h"

#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;

void oracle_set_num_threads(int n)
{
    g_threads = n;
}

#ifdef _OPENMP
#define ORACLE_PARALLEL_FOR _Pragma("omp parallel for schedule(dynamic, 64) num_threads(g_threads > 0 ? g_threads : omp_get_max_threads())")
#else
#define ORACLE_PARALLEL_FOR
#endif

/* ------------------------------------------------------------------------------------ */
/* AES-128, FIPS-197. S-box built from its definition (inverse in GF(2^8) + affine map). */
/* ------------------------------------------------------------------------------------ */

static uint8_t  SB[256];
static uint32_t TE0[256];

static uint8_t xtime8(uint8_t a)
{
    return (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1b : 0x00));
}

static uint8_t gf_mul(uint8_t a, uint8_t b)
{
    uint8_t r = 0;
    while (b)
    {
        if (b & 1) r ^= a;
        a = xtime8(a);
        b >>= 1;
    }
    return r;
}

static uint8_t rotl8(uint8_t x, int s)
{
    return (uint8_t)((x << s) | (x >> (8 - s)));
}

__attribute__((constructor)) static void oracle_aes_tables_init(void)
{
    for (int x = 0; x < 256; x++)
    {
        uint8_t inv = 0;
        if (x != 0)
        {
            /* x^254 = x^-1 in GF(2^8) */
            uint8_t r = 1, b = (uint8_t)x;
            int     e = 254;
            while (e)
            {
                if (e & 1) r = gf_mul(r, b);
                b = gf_mul(b, b);
                e >>= 1;
            }
            inv = r;
        }
        uint8_t s  = (uint8_t)(inv ^ rotl8(inv, 1) ^ rotl8(inv, 2) ^ rotl8(inv, 3) ^ rotl8(inv, 4) ^ 0x63);
        uint8_t s2 = xtime8(s);
        uint8_t s3 = (uint8_t)(s2 ^ s);
        SB[x]      = s;
        TE0[x]     = ((uint32_t)s2 << 24) | ((uint32_t)s << 16) | ((uint32_t)s << 8) | (uint32_t)s3;
    }
}

static inline uint32_t ror32(uint32_t x, int r)
{
    return (x >> r) | (x << (32 - r));
}

static inline uint32_t ld_be32(const uint8_t *p)
{
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}

static inline void st_be32(uint8_t *p, uint32_t v)
{
    p[0] = (uint8_t)(v >> 24);
    p[1] = (uint8_t)(v >> 16);
    p[2] = (uint8_t)(v >> 8);
    p[3] = (uint8_t)v;
}

typedef struct
{
    uint32_t rk[44];
} aes_ks_t;

/* Key schedule: src/impl/aes.h:170-200 (FIPS-197 5.2). */
static void aes_expand(aes_ks_t *ks, const uint8_t key[16])
{
    static const uint8_t RCON[10] = {0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1b, 0x36};
    for (int i = 0; i < 4; i++) ks->rk[i] = ld_be32(key + 4 * i);
    for (int i = 4; i < 44; i++)
    {
        uint32_t t = ks->rk[i - 1];
        if ((i & 3) == 0)
        {
            t = ((uint32_t)SB[(t >> 16) & 0xff] << 24) | ((uint32_t)SB[(t >> 8) & 0xff] << 16) |
                ((uint32_t)SB[t & 0xff] << 8) | (uint32_t)SB[t >> 24];
            t ^= (uint32_t)RCON[i / 4 - 1] << 24;
        }
        ks->rk[i] = ks->rk[i - 4] ^ t;
    }
}

/* Block encryption: src/impl/aes.h:207-272,280-302. */
static void aes_encrypt(const aes_ks_t *ks, const uint8_t in[16], uint8_t out[16])
{
    const uint32_t *rk = ks->rk;
    uint32_t        s0 = ld_be32(in) ^ rk[0], s1 = ld_be32(in + 4) ^ rk[1];
    uint32_t        s2 = ld_be32(in + 8) ^ rk[2], s3 = ld_be32(in + 12) ^ rk[3];
    for (int r = 1; r < 10; r++)
    {
        const uint32_t *k  = rk + 4 * r;
        uint32_t        t0 = TE0[s0 >> 24] ^ ror32(TE0[(s1 >> 16) & 0xff], 8) ^ ror32(TE0[(s2 >> 8) & 0xff], 16) ^
                      ror32(TE0[s3 & 0xff], 24) ^ k[0];
        uint32_t t1 = TE0[s1 >> 24] ^ ror32(TE0[(s2 >> 16) & 0xff], 8) ^ ror32(TE0[(s3 >> 8) & 0xff], 16) ^
                      ror32(TE0[s0 & 0xff], 24) ^ k[1];
        uint32_t t2 = TE0[s2 >> 24] ^ ror32(TE0[(s3 >> 16) & 0xff], 8) ^ ror32(TE0[(s0 >> 8) & 0xff], 16) ^
                      ror32(TE0[s1 & 0xff], 24) ^ k[2];
        uint32_t t3 = TE0[s3 >> 24] ^ ror32(TE0[(s0 >> 16) & 0xff], 8) ^ ror32(TE0[(s1 >> 8) & 0xff], 16) ^
                      ror32(TE0[s2 & 0xff], 24) ^ k[3];
        s0 = t0, s1 = t1, s2 = t2, s3 = t3;
    }
    const uint32_t *k = rk + 40;
#define LAST(a, b, c, d)                                                                                   \
    (((uint32_t)SB[(a) >> 24] << 24) | ((uint32_t)SB[((b) >> 16) & 0xff] << 16) |                          \
     ((uint32_t)SB[((c) >> 8) & 0xff] << 8) | (uint32_t)SB[(d) & 0xff])
    st_be32(out, LAST(s0, s1, s2, s3) ^ k[0]);
    st_be32(out + 4, LAST(s1, s2, s3, s0) ^ k[1]);
    st_be32(out + 8, LAST(s2, s3, s0, s1) ^ k[2]);
    st_be32(out + 12, LAST(s3, s0, s1, s2) ^ k[3]);
#undef LAST
}

void oracle_aes128_encrypt(const void *key16, const void *in16, void *out16)
{
    aes_ks_t ks;
    aes_expand(&ks, (const uint8_t *)key16);
    uint8_t tmp[16];
    aes_encrypt(&ks, (const uint8_t *)in16, tmp);
    memcpy(out16, tmp, 16);
}

/* G(s): AES_s over plaintext blocks first..first+nblk-1, block j = LE64(2j) || LE64(2j+1). */
static void prg(const uint64_t seed[2], int first, int nblk, uint64_t *out)
{
    aes_ks_t ks;
    aes_expand(&ks, (const uint8_t *)seed);
    for (int j = 0; j < nblk; j++)
    {
        uint64_t p[2] = {(uint64_t)(2 * (first + j)), (uint64_t)(2 * (first + j) + 1)};
        aes_encrypt(&ks, (const uint8_t *)p, (uint8_t *)(out + 2 * j));
    }
}

/* AES-CTR generator: src/cpu/prng.cpp:20-76. */
void oracle_prng_gen(const void *seed16, void *counter16, void *dst, size_t bytesNum)
{
    aes_ks_t ks;
    aes_expand(&ks, (const uint8_t *)seed16);
    uint64_t *ctr      = (uint64_t *)counter16;
    size_t    blockNum = bytesNum / 16, rem = bytesNum % 16;
    uint8_t  *d        = (uint8_t *)dst;
    for (size_t i = 0; i < blockNum; i++)
    {
        uint64_t c[2];
        c[0] = ctr[0] + i;
        c[1] = ctr[1] + (c[0] < ctr[0]);
        aes_encrypt(&ks, (const uint8_t *)c, d + 16 * i);
    }
    if (rem)
    {
        uint64_t c[2];
        uint8_t  buf[16];
        c[0] = ctr[0] + blockNum;
        c[1] = ctr[1] + (c[0] < ctr[0]);
        aes_encrypt(&ks, (const uint8_t *)c, buf);
        memcpy(d + 16 * blockNum, buf, rem);
        blockNum += 1;
    }
    ctr[0] = ctr[0] + blockNum;
    ctr[1] = ctr[1] + (ctr[0] < blockNum);
}

/* ------------------------------------------------------------------------------------ */
/* Ring helpers                                                                          */
/* ------------------------------------------------------------------------------------ */

static const uint64_t MASK_MSB63 = 0xFFFFFFFFFFFFFFFEULL;

static inline uint64_t esmask(size_t es)
{
    return es >= 8 ? ~0ULL : ((1ULL << (8 * es)) - 1);
}

/* modBits: src/impl/number.h:30-43 */
static inline uint64_t modbits(uint64_t x, size_t w)
{
    return w >= 64 ? x : (x & ((1ULL << w) - 1));
}

static inline uint64_t ld_el(const void *p, size_t i, size_t es)
{
    switch (es)
    {
        case 1: return ((const uint8_t *)p)[i];
        case 2: return ((const uint16_t *)p)[i];
        case 4: return ((const uint32_t *)p)[i];
        default: return ((const uint64_t *)p)[i];
    }
}

static inline void st_el(void *p, size_t i, size_t es, uint64_t v)
{
    switch (es)
    {
        case 1: ((uint8_t *)p)[i] = (uint8_t)v; break;
        case 2: ((uint16_t *)p)[i] = (uint16_t)v; break;
        case 4: ((uint32_t *)p)[i] = (uint32_t)v; break;
        default: ((uint64_t *)p)[i] = v; break;
    }
}

/* parityU64: src/impl/number.h:45-52 */
static inline int parity64(uint64_t x)
{
    return __builtin_parityll(x);
}

/* ------------------------------------------------------------------------------------ */
/* Value convert (DcfConvertCtx, src/impl/dcf.h:69-137; DpfConvertCtx src/impl/dpf.h:63-128) */
/* ------------------------------------------------------------------------------------ */

typedef struct
{
    uint8_t  buf[16];
    aes_ks_t ks;
    int      goff, ges, gsz, use_aes;
} conv_t;

static void conv_init(conv_t *c, const uint64_t seed[2], size_t groupSize, size_t bitWidth)
{
    c->gsz = (int)groupSize;
    c->ges = (int)((bitWidth + 7) / 8);
    if (c->ges * c->gsz <= 16)
    {
        memcpy(c->buf, seed, 16);
        c->use_aes = 0;
    }
    else
    {
        aes_expand(&c->ks, (const uint8_t *)seed);
        c->use_aes = 1;
    }
    c->goff = 0;
}

/* Bytes at or beyond 8 positions are shifted out of a 64-bit value (the CUDA build's
 * shift semantics); callers reduce to the element width. */
static uint64_t conv_next(conv_t *c)
{
    uint64_t r   = 0;
    int      off = c->goff * c->ges;
    for (int i = 0; i < c->ges; i++)
    {
        int idx = (off + i) % 16;
        if (c->use_aes && idx == 0)
        {
            uint64_t b[2] = {0, (uint64_t)c->goff};
            aes_encrypt(&c->ks, (const uint8_t *)b, c->buf);
        }
        if (i < 8) r |= (uint64_t)c->buf[idx] << (8 * i);
    }
    c->goff++;
    return r;
}

/* ------------------------------------------------------------------------------------ */
/* DCF (src/impl/dcf.h)                                                                  */
/* ------------------------------------------------------------------------------------ */

typedef struct
{
    uint8_t *sCW;   /* n x 16 bytes */
    uint8_t *vCW;   /* n*g elements */
    uint8_t *tLCW;  /* 1 element */
    uint8_t *tRCW;  /* 1 element */
    uint8_t *lastCW; /* g elements */
} dcf_key_t;

/* dcfKeySetPtr: src/impl/dcf.h:139-167 */
static void dcf_key_ptrs(dcf_key_t *k, const void *keyData, size_t n, size_t g, size_t es, size_t idx, size_t N)
{
    uint8_t *base = (uint8_t *)keyData;
    size_t   bstr = es * n * g + es + es + es * g;
    k->sCW        = base + idx * 16 * n;
    k->vCW        = base + N * 16 * n + idx * bstr;
    k->tLCW       = k->vCW + es * n * g;
    k->tRCW       = k->tLCW + es;
    k->lastCW     = k->tRCW + es;
}

static void dcf_keygen_one(const dcf_key_t *key, uint64_t alpha, const uint64_t *beta, const uint8_t *seed0,
                           const uint8_t *seed1, size_t n, size_t bo, size_t g, size_t es)
{
    /* dcfKeyGen: src/impl/dcf.h:187-368 */
    const uint64_t M = esmask(es);
    uint64_t       s0[2], s1[2];
    memcpy(s0, seed0, 16);
    memcpy(s1, seed1, 16);
    s0[0] &= MASK_MSB63;
    s1[0] &= MASK_MSB63;
    int       t0 = 0, t1 = 1;
    uint64_t  tl = 0, tr = 0;
    uint64_t *vAlpha = (uint64_t *)calloc(g, sizeof(uint64_t));
    uint64_t *vcw    = (uint64_t *)calloc(g, sizeof(uint64_t));
    conv_t    cv;
    for (size_t i = 0; i < n; i++)
    {
        size_t   bitShift = n - i - 1;
        uint64_t G0[8], G1[8];
        prg(s0, 0, 4, G0);
        prg(s1, 0, 4, G1);
        uint64_t *sL0 = G0 + 0, *vL0 = G0 + 2, *sR0 = G0 + 4, *vR0 = G0 + 6;
        uint64_t *sL1 = G1 + 0, *vL1 = G1 + 2, *sR1 = G1 + 4, *vR1 = G1 + 6;
        int       tL0 = (int)(sL0[0] & 1), tR0 = (int)(sR0[0] & 1);
        int       tL1 = (int)(sL1[0] & 1), tR1 = (int)(sR1[0] & 1);
        sL0[0] &= MASK_MSB63, sR0[0] &= MASK_MSB63, sL1[0] &= MASK_MSB63, sR1[0] &= MASK_MSB63;
        int keep = (int)((alpha >> bitShift) & 1), lose = 1 - keep;
        uint64_t *sLose0, *sLose1, *sKeep0, *sKeep1, *vLose0, *vLose1, *vKeep0, *vKeep1;
        if (lose == 0)
        {
            sLose0 = sL0, sLose1 = sL1, vLose0 = vL0, vLose1 = vL1;
            sKeep0 = sR0, sKeep1 = sR1, vKeep0 = vR0, vKeep1 = vR1;
        }
        else
        {
            sLose0 = sR0, sLose1 = sR1, vLose0 = vR0, vLose1 = vR1;
            sKeep0 = sL0, sKeep1 = sL1, vKeep0 = vL0, vKeep1 = vL1;
        }
        uint64_t sCW[2] = {sLose0[0] ^ sLose1[0], sLose0[1] ^ sLose1[1]};
        /* vCW <- (-1)^t1 (convert(vLose1) - convert(vLose0) - vAlpha) [+ (-1)^t1 beta if lose = L] */
        conv_init(&cv, vLose1, g, bo);
        for (size_t j = 0; j < g; j++) vcw[j] = conv_next(&cv);
        conv_init(&cv, vLose0, g, bo);
        for (size_t j = 0; j < g; j++) vcw[j] -= conv_next(&cv);
        for (size_t j = 0; j < g; j++)
        {
            vcw[j] -= vAlpha[j];
            if (t1) vcw[j] = 0 - vcw[j];
            if (lose == 0) vcw[j] += t1 ? (0 - beta[j]) : beta[j];
            vcw[j] &= M;
        }
        /* vAlpha += -convert(vKeep1) + convert(vKeep0) + (-1)^t1 vCW */
        conv_init(&cv, vKeep1, g, bo);
        for (size_t j = 0; j < g; j++) vAlpha[j] -= conv_next(&cv);
        conv_init(&cv, vKeep0, g, bo);
        for (size_t j = 0; j < g; j++) vAlpha[j] += conv_next(&cv);
        for (size_t j = 0; j < g; j++)
        {
            vAlpha[j] += t1 ? (0 - vcw[j]) : vcw[j];
            vAlpha[j] &= M;
            st_el(key->vCW, i * g + j, es, vcw[j]);
        }
        int tLCW = tL0 ^ tL1 ^ keep ^ 1;
        int tRCW = tR0 ^ tR1 ^ keep;
        memcpy(key->sCW + 16 * i, sCW, 16);
        tl |= (uint64_t)tLCW << i;
        tr |= (uint64_t)tRCW << i;
        s0[0] = t0 ? (sKeep0[0] ^ sCW[0]) : sKeep0[0];
        s0[1] = t0 ? (sKeep0[1] ^ sCW[1]) : sKeep0[1];
        s1[0] = t1 ? (sKeep1[0] ^ sCW[0]) : sKeep1[0];
        s1[1] = t1 ? (sKeep1[1] ^ sCW[1]) : sKeep1[1];
        if (keep == 0)
        {
            t0 = tLCW ? (tL0 ^ t0) : tL0;
            t1 = tLCW ? (tL1 ^ t1) : tL1;
        }
        else
        {
            t0 = tRCW ? (tR0 ^ t0) : tR0;
            t1 = tRCW ? (tR1 ^ t1) : tR1;
        }
    }
    st_el(key->tLCW, 0, es, tl);
    st_el(key->tRCW, 0, es, tr);
    /* CW(n+1) <- (-1)^t1 (convert(s1) - convert(s0) - vAlpha) */
    conv_t c1, c0;
    conv_init(&c1, s1, g, bo);
    conv_init(&c0, s0, g, bo);
    for (size_t j = 0; j < g; j++)
    {
        uint64_t last = 0 - vAlpha[j];
        last += conv_next(&c1);
        last -= conv_next(&c0);
        if (t1) last = 0 - last;
        st_el(key->lastCW, j, es, last & M);
    }
    free(vAlpha);
    free(vcw);
}

/* dcfEval: src/impl/dcf.h:370-491 (no prefix cache; the cache never changes results). */
static void dcf_eval_one(uint64_t *out, const dcf_key_t *key, uint64_t x, const uint8_t *seed, int party, size_t n,
                         size_t bo, size_t g, size_t es)
{
    const uint64_t M = esmask(es);
    uint64_t       s[2];
    memcpy(s, seed, 16);
    s[0] &= MASK_MSB63;
    int t = party;
    x     = modbits(x, n);
    for (size_t j = 0; j < g; j++) out[j] = 0;
    uint64_t tl = ld_el(key->tLCW, 0, es), tr = ld_el(key->tRCW, 0, es);
    conv_t   cv;
    for (size_t i = 0; i < n; i++)
    {
        size_t   bitShift = n - i - 1;
        uint64_t G[8];
        prg(s, 0, 4, G);
        uint64_t *sL = G + 0, *vL = G + 2, *sR = G + 4, *vR = G + 6;
        int       tL = (int)(sL[0] & 1), tR = (int)(sR[0] & 1);
        sL[0] &= MASK_MSB63;
        sR[0] &= MASK_MSB63;
        if (t)
        {
            uint64_t cw[2];
            memcpy(cw, key->sCW + 16 * i, 16);
            sL[0] ^= cw[0], sL[1] ^= cw[1], sR[0] ^= cw[0], sR[1] ^= cw[1];
            tL ^= (int)((tl >> i) & 1);
            tR ^= (int)((tr >> i) & 1);
        }
        int xi = (int)((x >> bitShift) & 1);
        int tp = t;
        if (xi == 0)
        {
            conv_init(&cv, vL, g, bo);
            s[0] = sL[0], s[1] = sL[1], t = tL;
        }
        else
        {
            conv_init(&cv, vR, g, bo);
            s[0] = sR[0], s[1] = sR[1], t = tR;
        }
        for (size_t j = 0; j < g; j++)
        {
            uint64_t v = conv_next(&cv) + (tp ? ld_el(key->vCW, i * g + j, es) : 0);
            out[j] += party ? (0 - v) : v;
        }
    }
    conv_init(&cv, s, g, bo);
    for (size_t j = 0; j < g; j++)
    {
        uint64_t v = conv_next(&cv) + (t ? ld_el(key->lastCW, j, es) : 0);
        out[j] += party ? (0 - v) : v;
        out[j] &= M;
    }
}

/* Task loops: src/kernel/dcf.h:73-91,165-191 */
void oracle_dcfKeyGen(void *key, const void *alpha, const void *beta, const void *seed0, const void *seed1,
                      size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *b = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        for (size_t j = 0; j < groupSize; j++) b[j] = beta ? ld_el(beta, i * groupSize + j, elementSize) : (j == 0);
        dcf_keygen_one(&k, ld_el(alpha, i, elementSize), b, (const uint8_t *)seed0 + 16 * i,
                       (const uint8_t *)seed1 + 16 * i, bitWidthIn, bitWidthOut, groupSize, elementSize);
        free(b);
    }
}

void oracle_dcfEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                    size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *o = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        dcf_eval_one(o, &k, ld_el(maskedX, i, elementSize), (const uint8_t *)seed + 16 * i, partyId, bitWidthIn,
                     bitWidthOut, groupSize, elementSize);
        for (size_t j = 0; j < groupSize; j++) st_el(sharedOut, i * groupSize + j, elementSize, o[j]);
        free(o);
    }
}

/* ------------------------------------------------------------------------------------ */
/* DPF (src/impl/dpf.h)                                                                  */
/* ------------------------------------------------------------------------------------ */

typedef struct
{
    uint8_t *sCW, *tLCW, *tRCW, *lastCW;
} dpf_key_t;

/* dpfKeySetPtr: src/impl/dpf.h:130-156 */
static void dpf_key_ptrs(dpf_key_t *k, const void *keyData, size_t n, size_t g, size_t es, size_t idx, size_t N)
{
    uint8_t *base = (uint8_t *)keyData;
    k->sCW        = base + idx * 16 * n;
    k->tLCW       = base + N * 16 * n + idx * (es + es + es * g);
    k->tRCW       = k->tLCW + es;
    k->lastCW     = k->tRCW + es;
}

/* dpfKeyGen: src/impl/dpf.h:172-288. Note the convert is initialised as init(s, bo, g)
 * (src/impl/dpf.h:278,283): byte width ceil(g/8), threshold on ceil(g/8)*bo. */
static void dpf_keygen_one(const dpf_key_t *key, uint64_t alpha, const uint64_t *beta, const uint8_t *seed0,
                           const uint8_t *seed1, size_t n, size_t bo, size_t g, size_t es)
{
    const uint64_t M = esmask(es);
    uint64_t       s0[2], s1[2];
    memcpy(s0, seed0, 16);
    memcpy(s1, seed1, 16);
    s0[0] &= MASK_MSB63;
    s1[0] &= MASK_MSB63;
    int      t0 = 0, t1 = 1;
    uint64_t tl = 0, tr = 0;
    for (size_t i = 0; i < n; i++)
    {
        size_t   bitShift = n - i - 1;
        uint64_t G0[4], G1[4];
        prg(s0, 0, 2, G0);
        prg(s1, 0, 2, G1);
        uint64_t *sL0 = G0, *sR0 = G0 + 2, *sL1 = G1, *sR1 = G1 + 2;
        int       tL0 = (int)(sL0[0] & 1), tR0 = (int)(sR0[0] & 1);
        int       tL1 = (int)(sL1[0] & 1), tR1 = (int)(sR1[0] & 1);
        sL0[0] &= MASK_MSB63, sR0[0] &= MASK_MSB63, sL1[0] &= MASK_MSB63, sR1[0] &= MASK_MSB63;
        int       keep = (int)((alpha >> bitShift) & 1), lose = 1 - keep;
        uint64_t *sLose0 = lose == 0 ? sL0 : sR0, *sLose1 = lose == 0 ? sL1 : sR1;
        uint64_t *sKeep0 = lose == 0 ? sR0 : sL0, *sKeep1 = lose == 0 ? sR1 : sL1;
        uint64_t  sCW[2] = {sLose0[0] ^ sLose1[0], sLose0[1] ^ sLose1[1]};
        int       tLCW = tL0 ^ tL1 ^ keep ^ 1, tRCW = tR0 ^ tR1 ^ keep;
        memcpy(key->sCW + 16 * i, sCW, 16);
        tl |= (uint64_t)tLCW << i;
        tr |= (uint64_t)tRCW << i;
        s0[0] = t0 ? (sKeep0[0] ^ sCW[0]) : sKeep0[0];
        s0[1] = t0 ? (sKeep0[1] ^ sCW[1]) : sKeep0[1];
        s1[0] = t1 ? (sKeep1[0] ^ sCW[0]) : sKeep1[0];
        s1[1] = t1 ? (sKeep1[1] ^ sCW[1]) : sKeep1[1];
        if (keep == 0)
        {
            t0 = tLCW ? (tL0 ^ t0) : tL0;
            t1 = tLCW ? (tL1 ^ t1) : tL1;
        }
        else
        {
            t0 = tRCW ? (tR0 ^ t0) : tR0;
            t1 = tRCW ? (tR1 ^ t1) : tR1;
        }
    }
    st_el(key->tLCW, 0, es, tl);
    st_el(key->tRCW, 0, es, tr);
    conv_t c0, c1;
    conv_init(&c0, s0, bo, g);
    conv_init(&c1, s1, bo, g);
    for (size_t j = 0; j < g; j++)
    {
        uint64_t a    = conv_next(&c0);
        uint64_t b    = conv_next(&c1);
        uint64_t last = beta[j] - a + b;
        if (t1) last = 0 - last;
        st_el(key->lastCW, j, es, last & M);
    }
}

/* dpfEval: src/impl/dpf.h:290-380 */
static void dpf_eval_one(uint64_t *out, const dpf_key_t *key, uint64_t x, const uint8_t *seed, int party, size_t n,
                         size_t bo, size_t g, size_t es)
{
    const uint64_t M = esmask(es);
    uint64_t       s[2];
    memcpy(s, seed, 16);
    s[0] &= MASK_MSB63;
    int t = party;
    x     = modbits(x, n);
    uint64_t tl = ld_el(key->tLCW, 0, es), tr = ld_el(key->tRCW, 0, es);
    for (size_t i = 0; i < n; i++)
    {
        size_t   bitShift = n - i - 1;
        uint64_t G[4];
        prg(s, 0, 2, G);
        uint64_t *sL = G, *sR = G + 2;
        int       tL = (int)(sL[0] & 1), tR = (int)(sR[0] & 1);
        sL[0] &= MASK_MSB63;
        sR[0] &= MASK_MSB63;
        if (t)
        {
            uint64_t cw[2];
            memcpy(cw, key->sCW + 16 * i, 16);
            sL[0] ^= cw[0], sL[1] ^= cw[1], sR[0] ^= cw[0], sR[1] ^= cw[1];
            tL ^= (int)((tl >> i) & 1);
            tR ^= (int)((tr >> i) & 1);
        }
        if (((x >> bitShift) & 1) == 0)
            s[0] = sL[0], s[1] = sL[1], t = tL;
        else
            s[0] = sR[0], s[1] = sR[1], t = tR;
    }
    conv_t cv;
    conv_init(&cv, s, bo, g);
    for (size_t j = 0; j < g; j++)
    {
        uint64_t v = conv_next(&cv) + (t ? ld_el(key->lastCW, j, es) : 0);
        out[j]     = (party ? (0 - v) : v) & M;
    }
}

/* Task loops: src/kernel/dpf.h:76-91,162-179,253-276,472-496 */
void oracle_dpfKeyGen(void *key, const void *alpha, const void *beta, const void *seed0, const void *seed1,
                      size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dpf_key_t k;
        dpf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *b = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        for (size_t j = 0; j < groupSize; j++) b[j] = beta ? ld_el(beta, i * groupSize + j, elementSize) : (j == 0);
        dpf_keygen_one(&k, ld_el(alpha, i, elementSize), b, (const uint8_t *)seed0 + 16 * i,
                       (const uint8_t *)seed1 + 16 * i, bitWidthIn, bitWidthOut, groupSize, elementSize);
        free(b);
    }
}

void oracle_dpfEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                    size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dpf_key_t k;
        dpf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *o = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        dpf_eval_one(o, &k, ld_el(maskedX, i, elementSize), (const uint8_t *)seed + 16 * i, partyId, bitWidthIn,
                     bitWidthOut, groupSize, elementSize);
        for (size_t j = 0; j < groupSize; j++) st_el(sharedOut, i * groupSize + j, elementSize, o[j]);
        free(o);
    }
}

void oracle_dpfEvalAll(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                       size_t bitWidthIn, size_t bitWidthOut, size_t groupSize, size_t elementSize,
                       size_t elementNum)
{
    size_t size = (size_t)1 << bitWidthIn;
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dpf_key_t k;
        dpf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *o  = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        size_t    mx = (size_t)ld_el(maskedX, i, elementSize);
        for (size_t j = 0; j < size; j++)
        {
            size_t kk = groupSize * ((mx - j) % size);
            dpf_eval_one(o, &k, (uint64_t)j, (const uint8_t *)seed + 16 * i, partyId, bitWidthIn, bitWidthOut,
                         groupSize, elementSize);
            for (size_t q = 0; q < groupSize; q++) st_el(sharedOut, size * i * groupSize + kk + q, elementSize, o[q]);
        }
        free(o);
    }
}

void oracle_dpfEvalMulti(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                         const void *point, size_t pointNum, size_t bitWidthIn, size_t bitWidthOut, size_t groupSize,
                         size_t elementSize, size_t elementNum)
{
    const uint64_t M = esmask(elementSize);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dpf_key_t k;
        dpf_key_ptrs(&k, key, bitWidthIn, groupSize, elementSize, i, elementNum);
        uint64_t *o = (uint64_t *)malloc(groupSize * sizeof(uint64_t));
        for (size_t j = 0; j < pointNum; j++)
        {
            uint64_t x = (ld_el(maskedX, i, elementSize) - ld_el(point, j, elementSize)) & M;
            dpf_eval_one(o, &k, x, (const uint8_t *)seed + 16 * i, partyId, bitWidthIn, bitWidthOut, groupSize,
                         elementSize);
            for (size_t q = 0; q < groupSize; q++)
                st_el(sharedOut, pointNum * i * groupSize + j * groupSize + q, elementSize, o[q]);
        }
        free(o);
    }
}

/* ------------------------------------------------------------------------------------ */
/* Grotto (src/impl/grotto.h)                                                            */
/* ------------------------------------------------------------------------------------ */

typedef struct
{
    uint8_t *sCW;    /* (n-6) x 16 bytes */
    uint8_t *lastCW; /* uint64 */
    uint8_t *tLCW, *tRCW;
} grotto_key_t;

/* grottoKeySetPtr: src/impl/grotto.h:53-79 */
static void grotto_key_ptrs(grotto_key_t *k, const void *keyData, size_t n, size_t es, size_t idx, size_t N)
{
    uint8_t *base = (uint8_t *)keyData;
    k->sCW        = base + idx * 16 * (n - 6);
    k->lastCW     = base + N * 16 * (n - 6) + idx * 8;
    k->tLCW       = base + N * 16 * (n - 6) + N * 8 + idx * es * 2;
    k->tRCW       = k->tLCW + es;
}

/* grottoKeyGen: src/impl/grotto.h:111-205 */
static void grotto_keygen_one(const grotto_key_t *key, uint64_t alpha, const uint8_t *seed0, const uint8_t *seed1,
                              size_t n, size_t es)
{
    uint64_t s0[2], s1[2];
    memcpy(s0, seed0, 16);
    memcpy(s1, seed1, 16);
    s0[0] &= MASK_MSB63;
    s1[0] &= MASK_MSB63;
    int      t0 = 0, t1 = 1;
    uint64_t tl = 0, tr = 0;
    for (size_t i = 0; i + 6 < n; i++)
    {
        size_t   bitShift = n - i - 1;
        uint64_t G0[4], G1[4];
        prg(s0, 0, 2, G0);
        prg(s1, 0, 2, G1);
        uint64_t *sL0 = G0, *sR0 = G0 + 2, *sL1 = G1, *sR1 = G1 + 2;
        int       tL0 = (int)(sL0[0] & 1), tR0 = (int)(sR0[0] & 1);
        int       tL1 = (int)(sL1[0] & 1), tR1 = (int)(sR1[0] & 1);
        sL0[0] &= MASK_MSB63, sR0[0] &= MASK_MSB63, sL1[0] &= MASK_MSB63, sR1[0] &= MASK_MSB63;
        int      keep = (int)((alpha >> bitShift) & 1), lose = 1 - keep;
        uint64_t cw[2];
        cw[0] = lose == 0 ? (sL0[0] ^ sL1[0]) : (sR0[0] ^ sR1[0]);
        cw[1] = lose == 0 ? (sL0[1] ^ sL1[1]) : (sR0[1] ^ sR1[1]);
        memcpy(key->sCW + 16 * i, cw, 16);
        int tLCW = tL0 ^ tL1 ^ lose, tRCW = tR0 ^ tR1 ^ keep;
        tl |= (uint64_t)tLCW << i;
        tr |= (uint64_t)tRCW << i;
        uint64_t *k0 = keep == 0 ? sL0 : sR0, *k1 = keep == 0 ? sL1 : sR1;
        s0[0]        = t0 ? (k0[0] ^ cw[0]) : k0[0];
        s0[1]        = t0 ? (k0[1] ^ cw[1]) : k0[1];
        s1[0]        = t1 ? (k1[0] ^ cw[0]) : k1[0];
        s1[1]        = t1 ? (k1[1] ^ cw[1]) : k1[1];
        t0           = t0 == 0 ? (keep == 0 ? tL0 : tR0) : (keep == 0 ? (tL0 ^ tLCW) : (tR0 ^ tRCW));
        t1           = t1 == 0 ? (keep == 0 ? tL1 : tR1) : (keep == 0 ? (tL1 ^ tLCW) : (tR1 ^ tRCW));
    }
    st_el(key->tLCW, 0, es, tl);
    st_el(key->tRCW, 0, es, tr);
    uint64_t last = s0[1] ^ s1[1] ^ (1ULL << (alpha & 63));
    memcpy(key->lastCW, &last, 8);
}

/* Walk from the root to the leaf of x (n-6 levels), one child block per level
 * (src/impl/grotto.h:241-278 and 321-375). Returns the leaf word u and the
 * right-turn path parity; with equalBound the early exit of src/impl/grotto.h:326-334
 * is taken and *early set. */
static uint64_t grotto_walk(const grotto_key_t *key, uint64_t x, const uint8_t *seed, int party, size_t n, size_t es,
                            int equalBound, int *parityOut, int *early)
{
    uint64_t s[2];
    memcpy(s, seed, 16);
    s[0] &= MASK_MSB63;
    int      t = party, parity = 0;
    uint64_t tl = ld_el(key->tLCW, 0, es), tr = ld_el(key->tRCW, 0, es);
    *early      = 0;
    for (size_t i = 0; i + 6 < n; i++)
    {
        size_t bitShift = n - 1 - i;
        if (equalBound)
        {
            uint64_t mask = modbits(~0ULL, n - i);
            if ((x & mask) == 0)
            {
                *early     = 1;
                *parityOut = parity;
                return 0;
            }
        }
        int      b = (int)((x >> bitShift) & 1);
        uint64_t c[2];
        prg(s, b, 1, c);
        int ti = (int)(c[0] & 1);
        c[0] &= MASK_MSB63;
        uint64_t cw[2];
        memcpy(cw, key->sCW + 16 * i, 16);
        s[0]       = t ? (c[0] ^ cw[0]) : c[0];
        s[1]       = t ? (c[1] ^ cw[1]) : c[1];
        uint64_t w = b ? tr : tl;
        int      nt = t ? (ti ^ (int)((w >> i) & 1)) : ti;
        parity     = b ? (parity ^ (t ^ nt)) : parity;
        t          = nt;
    }
    uint64_t last;
    memcpy(&last, key->lastCW, 8);
    *parityOut = parity;
    return t ? (s[1] ^ last) : s[1];
}

/* grottoEqEval: src/impl/grotto.h:207-282 */
static uint64_t grotto_eq_one(const grotto_key_t *key, uint64_t x, const uint8_t *seed, int party, size_t n, size_t es)
{
    int p, e;
    x          = modbits(x, n);
    uint64_t u = grotto_walk(key, x, seed, party, n, es, 0, &p, &e);
    return (u >> (x & 63)) & 1;
}

/* grottoEval: src/impl/grotto.h:284-391 */
static uint64_t grotto_eval_one(const grotto_key_t *key, uint64_t x, const uint8_t *seed, int party, size_t n,
                                size_t es, int equalBound)
{
    int parity, early;
    x          = modbits(x, n);
    uint64_t u = grotto_walk(key, x, seed, party, n, es, equalBound, &parity, &early);
    if (early) return (uint64_t)(parity ^ party);
    unsigned prefixLen = (unsigned)(x & 63);
    if (equalBound)
    {
        if (prefixLen != 0) parity ^= parity64(u & (~0ULL >> (64 - prefixLen)));
    }
    else
    {
        parity ^= parity64(u & (~0ULL >> (63 - prefixLen)));
    }
    return (uint64_t)(parity ^ party);
}

void oracle_grottoKeyGen(void *key, const void *alpha, const void *seed0, const void *seed1, size_t bitWidthIn,
                         size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, bitWidthIn, elementSize, i, elementNum);
        grotto_keygen_one(&k, ld_el(alpha, i, elementSize), (const uint8_t *)seed0 + 16 * i,
                          (const uint8_t *)seed1 + 16 * i, bitWidthIn, elementSize);
    }
}

void oracle_grottoEqEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                         size_t bitWidthIn, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, bitWidthIn, elementSize, i, elementNum);
        st_el(sharedOut, i, elementSize,
              grotto_eq_one(&k, ld_el(maskedX, i, elementSize), (const uint8_t *)seed + 16 * i, partyId, bitWidthIn,
                            elementSize));
    }
}

void oracle_grottoEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int equalBound,
                       int partyId, size_t bitWidthIn, size_t elementSize, size_t elementNum)
{
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, bitWidthIn, elementSize, i, elementNum);
        st_el(sharedOut, i, elementSize,
              grotto_eval_one(&k, ld_el(maskedX, i, elementSize), (const uint8_t *)seed + 16 * i, partyId,
                              bitWidthIn, elementSize, equalBound));
    }
}

/* grottoMICEval: src/impl/grotto.h:393-447 */
void oracle_grottoMICEval(void *sharedOut, const void *maskedX, const void *key, const void *seed, int partyId,
                          const void *leftEndpoints, const void *rightEndpoints, size_t intervalNum, size_t bitWidthIn,
                          size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, n, es, i, elementNum);
        const uint8_t *sd = (const uint8_t *)seed + 16 * i;
        uint64_t       x  = ld_el(maskedX, i, es);
        uint64_t       sp = 0, sq = 0;
        for (size_t q = 0; q < intervalNum; q++)
        {
            uint64_t L  = ld_el(leftEndpoints, q, es), R = ld_el(rightEndpoints, q, es);
            uint64_t xP = modbits((x - (L - 1)) & M, n);
            uint64_t xQ = modbits((x - R) & M, n);
            if (q > 0 && L == modbits((ld_el(rightEndpoints, q - 1, es) + 1) & M, n))
                sp = sq;
            else
                sp = grotto_eval_one(&k, xP, sd, partyId, n, es, 1);
            sq = grotto_eval_one(&k, xQ, sd, partyId, n, es, 1);
            st_el(sharedOut, intervalNum * i + q, es, (sp ^ sq) ^ (uint64_t)((xQ >= xP) ? partyId : 0));
        }
    }
}

/* grottoIntervalLutEval: src/impl/grotto.h:449-545 */
void oracle_grottoIntervalLutEval(void *sharedOutE, void *sharedOutT, const void *maskedX, const void *key,
                                  const void *seed, int partyId, const void *leftEndpoints, const void *rightEndpoints,
                                  const void *lookUpTable, size_t lutNum, size_t intervalNum, size_t bitWidthIn,
                                  size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn;
    const uint64_t M  = esmask(es);
    if (intervalNum == 0) return;
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, n, es, i, elementNum);
        const uint8_t *sd = (const uint8_t *)seed + 16 * i;
        uint64_t       x  = ld_el(maskedX, i, es);
        uint64_t       sp = 0, sq = 0, E = 0;
        uint64_t      *T  = (uint64_t *)calloc(lutNum ? lutNum : 1, sizeof(uint64_t));
        for (size_t q = 0; q < intervalNum; q++)
        {
            uint64_t L  = ld_el(leftEndpoints, q, es), R = ld_el(rightEndpoints, q, es);
            uint64_t xP = modbits((x - (L - 1)) & M, n);
            uint64_t xQ = modbits((x - R) & M, n);
            if (q > 0 && L == modbits((ld_el(rightEndpoints, q - 1, es) + 1) & M, n))
                sp = sq;
            else
                sp = grotto_eval_one(&k, xP, sd, partyId, n, es, 1);
            sq           = grotto_eval_one(&k, xQ, sd, partyId, n, es, 1);
            uint64_t tmp = ((sp ^ sq) ^ (uint64_t)((xQ >= xP) ? partyId : 0)) & 1;
            E += tmp;
            for (size_t j = 0; j < lutNum; j++) T[j] += tmp * ld_el(lookUpTable, q + j * intervalNum, es);
        }
        if (partyId)
        {
            E = 0 - E;
            for (size_t j = 0; j < lutNum; j++) T[j] = 0 - T[j];
        }
        st_el(sharedOutE, i, es, E & M);
        for (size_t j = 0; j < lutNum; j++) st_el(sharedOutT, i * lutNum + j, es, T[j] & M);
        free(T);
    }
}

/* Full-domain rows: the per-x reference evaluations above, packed LSB first into bytes. */
void oracle_grottoEqEvalAll(void *outBits, const void *key, const void *seed, int partyId, size_t bitWidthIn,
                            size_t elementSize, size_t elementNum)
{
    const size_t dom = (size_t)1 << bitWidthIn;
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, bitWidthIn, elementSize, i, elementNum);
        uint8_t *row = (uint8_t *)outBits + i * (dom / 8);
        memset(row, 0, dom / 8);
        for (size_t x = 0; x < dom; x++)
            if (grotto_eq_one(&k, x, (const uint8_t *)seed + 16 * i, partyId, bitWidthIn, elementSize))
                row[x >> 3] |= (uint8_t)(1u << (x & 7));
    }
}

void oracle_grottoLeEvalAll(void *outBits, const void *key, const void *seed, int partyId, size_t bitWidthIn,
                            size_t elementSize, size_t elementNum)
{
    const size_t dom = (size_t)1 << bitWidthIn;
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t       i = (size_t)ii;
        grotto_key_t k;
        grotto_key_ptrs(&k, key, bitWidthIn, elementSize, i, elementNum);
        uint8_t *row = (uint8_t *)outBits + i * (dom / 8);
        memset(row, 0, dom / 8);
        for (size_t x = 0; x < dom; x++)
            if (grotto_eval_one(&k, x, (const uint8_t *)seed + 16 * i, partyId, bitWidthIn, elementSize, 1))
                row[x >> 3] |= (uint8_t)(1u << (x & 7));
    }
}

/* ------------------------------------------------------------------------------------ */
/* DCF-based MIC (src/impl/mic.h)                                                        */
/* ------------------------------------------------------------------------------------ */

/* dcfMICKeyGen: src/impl/mic.h:9-41 */
void oracle_dcfMICKeyGen(void *key, void *z, const void *alpha, const void *seed0, const void *seed1,
                         const void *leftEndpoints, const void *rightEndpoints, size_t intervalNum, size_t bitWidthIn,
                         size_t bitWidthOut, size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, n, 1, es, i, elementNum);
        uint64_t a   = ld_el(alpha, i, es);
        uint64_t one = 1;
        dcf_keygen_one(&k, (a - 1) & M, &one, (const uint8_t *)seed0 + 16 * i, (const uint8_t *)seed1 + 16 * i, n,
                       bitWidthOut, 1, es);
        uint64_t MAX = modbits(M, n);
        for (size_t q = 0; q < intervalNum; q++)
        {
            uint64_t L = ld_el(leftEndpoints, q, es), R = ld_el(rightEndpoints, q, es);
            uint64_t qPrime = modbits((R + 1) & M, n), alphaP = modbits((L + a) & M, n);
            uint64_t alphaQ = modbits((R + a) & M, n), alphaQPrime = modbits((R + 1 + a) & M, n);
            uint64_t pi     = modbits(L, n);
            long long zz    = (long long)(alphaP > alphaQ) - (long long)(alphaP > pi) +
                           (long long)(alphaQPrime > qPrime) + (long long)(alphaQ == MAX);
            st_el(z, intervalNum * i + q, es, (uint64_t)zz & M);
        }
    }
}

/* dcfMICEval: src/impl/mic.h:43-109 */
void oracle_dcfMICEval(void *sharedOut, const void *maskedX, const void *key, const void *sharedZ, const void *seed,
                       int partyId, const void *leftEndpoints, const void *rightEndpoints, size_t intervalNum,
                       size_t bitWidthIn, size_t bitWidthOut, size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, n, 1, es, i, elementNum);
        const uint8_t *sd = (const uint8_t *)seed + 16 * i;
        uint64_t       x  = modbits(ld_el(maskedX, i, es), n);
        uint64_t       sp = 0, sq = 0;
        for (size_t q = 0; q < intervalNum; q++)
        {
            uint64_t L = ld_el(leftEndpoints, q, es), R = ld_el(rightEndpoints, q, es);
            uint64_t qPrime  = modbits((R + 1) & M, n);
            uint64_t xP      = modbits((x - 1 - L) & M, n);
            uint64_t xQPrime = modbits((x - 1 - qPrime) & M, n);
            uint64_t p       = modbits(L, n);
            if (q > 0 && L == modbits((ld_el(rightEndpoints, q - 1, es) + 1) & M, n))
                sp = sq;
            else
                dcf_eval_one(&sp, &k, xP, sd, partyId, n, bitWidthOut, 1, es);
            dcf_eval_one(&sq, &k, xQPrime, sd, partyId, n, bitWidthOut, 1, es);
            uint64_t o = sq - sp + ld_el(sharedZ, intervalNum * i + q, es);
            if (partyId == 1) o += (uint64_t)((long long)(x > p) - (long long)(x > qPrime));
            st_el(sharedOut, intervalNum * i + q, es, o & M);
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* DCF spline (src/impl/spline.h)                                                        */
/* ------------------------------------------------------------------------------------ */

/* splineShiftPolynomialCoefficients: src/impl/spline.h:89-117 */
static void spline_shift(uint64_t *out, const void *coeffs, size_t cOff, uint64_t shift, size_t d, size_t bo,
                         size_t es)
{
    const uint64_t M        = esmask(es);
    uint64_t       negShift = modbits((0 - shift) & M, bo);
    for (size_t i = 0; i <= d; i++) out[i] = 0;
    for (size_t i = d + 1; i > 0; --i)
    {
        uint64_t c = ld_el(coeffs, cOff + i - 1, es);
        for (size_t j = d; j > 0; --j) out[j] = (out[j - 1] + out[j] * negShift) & M;
        out[0] = (out[0] * negShift + c) & M;
    }
    for (size_t i = 0; i <= d; i++) out[i] = modbits(out[i], bo);
}

/* dcfSplineKeyGen: src/impl/spline.h:137-184 */
void oracle_dcfSplineKeyGen(void *key, void *e, void *beta, const void *alpha, const void *seed0, const void *seed1,
                            const void *coefficients, size_t degree, const void *leftEndpoints,
                            const void *rightEndpoints, size_t intervalNum, size_t bitWidthIn, size_t bitWidthOut,
                            size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn, bo = bitWidthOut;
    const size_t   cn = degree + 1, g = intervalNum * cn;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, n, g, es, i, elementNum);
        uint64_t  a = ld_el(alpha, i, es);
        uint64_t *b = (uint64_t *)malloc(g * sizeof(uint64_t));
        for (size_t q = 0; q < intervalNum; q++) spline_shift(b + q * cn, coefficients, q * cn, a, degree, bo, es);
        for (size_t j = 0; j < g; j++) st_el(beta, g * i + j, es, b[j]);
        dcf_keygen_one(&k, (a - 1) & M, b, (const uint8_t *)seed0 + 16 * i, (const uint8_t *)seed1 + 16 * i, n, bo,
                       g, es);
        uint64_t maxValue = modbits(M, n);
        for (size_t q = 0; q < intervalNum; q++)
        {
            uint64_t L  = modbits(ld_el(leftEndpoints, q, es), n);
            uint64_t R  = modbits(ld_el(rightEndpoints, q, es), n);
            uint64_t Rp = modbits((R + 1) & M, n);
            uint64_t aL = modbits((L + a) & M, n), aR = modbits((R + a) & M, n), aRp = modbits((Rp + a) & M, n);
            long long corr = (long long)(aL > aR) - (long long)(aL > L) + (long long)(aRp > Rp) +
                             (long long)(aR == maxValue);
            for (size_t j = 0; j < cn; j++)
                st_el(e, g * i + q * cn + j, es, modbits(((uint64_t)corr * b[q * cn + j]) & M, bo));
        }
        free(b);
    }
}

/* dcfSplineEval: src/impl/spline.h:186-253 */
void oracle_dcfSplineEval(void *sharedOut, const void *maskedX, const void *key, const void *sharedE,
                          const void *sharedBeta, const void *seed, int partyId, const void *leftEndpoints,
                          const void *rightEndpoints, size_t intervalNum, size_t degree, size_t bitWidthIn,
                          size_t bitWidthOut, size_t elementSize, size_t elementNum)
{
    const size_t   es = elementSize, n = bitWidthIn, bo = bitWidthOut;
    const size_t   cn = degree + 1, g = intervalNum * cn;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t    i = (size_t)ii;
        dcf_key_t k;
        dcf_key_ptrs(&k, key, n, g, es, i, elementNum);
        const uint8_t *sd  = (const uint8_t *)seed + 16 * i;
        uint64_t       x   = modbits(ld_el(maskedX, i, es), n);
        uint64_t      *cur = (uint64_t *)malloc(g * sizeof(uint64_t));
        uint64_t      *nxt = (uint64_t *)malloc(g * sizeof(uint64_t));
        uint64_t      *acc = (uint64_t *)calloc(cn, sizeof(uint64_t));
        if (intervalNum == 0)
        {
            st_el(sharedOut, i, es, 0);
        }
        else
        {
            for (size_t q = 0; q < intervalNum; q++)
            {
                uint64_t L  = modbits(ld_el(leftEndpoints, q, es), n);
                uint64_t R  = modbits(ld_el(rightEndpoints, q, es), n);
                uint64_t Rp = modbits((R + 1) & M, n);
                if (q > 0 && modbits((ld_el(rightEndpoints, q - 1, es) + 1) & M, n) == L)
                    memcpy(cur, nxt, g * sizeof(uint64_t));
                else
                    dcf_eval_one(cur, &k, (x - 1 - L) & M, sd, partyId, n, bo, g, es);
                dcf_eval_one(nxt, &k, (x - 1 - Rp) & M, sd, partyId, n, bo, g, es);
                uint64_t cx = (uint64_t)((long long)(x > L) - (long long)(x > Rp));
                for (size_t j = 0; j < cn; j++)
                {
                    uint64_t b = ld_el(sharedBeta, g * i + q * cn + j, es);
                    uint64_t w = cx * b - cur[q * cn + j] + nxt[q * cn + j] + ld_el(sharedE, g * i + q * cn + j, es);
                    acc[j]     = (acc[j] + w) & M;
                }
            }
            /* splineEvaluatePolynomial: src/impl/spline.h:119-135 */
            uint64_t r = 0, p = 1;
            for (size_t j = 0; j <= degree; j++)
            {
                r = (r + acc[j] * p) & M;
                p = (p * x) & M;
            }
            st_el(sharedOut, i, es, modbits(r, bo));
        }
        free(cur);
        free(nxt);
        free(acc);
    }
}

/* ------------------------------------------------------------------------------------ */
/* OTTT / one-hot truth table (src/impl/ottt.h)                                          */
/* ------------------------------------------------------------------------------------ */

/* otttKeyGen: src/impl/ottt.h:15-24 (XORs the one-hot bit of alpha into the key row). */
void oracle_otttKeyGen(void *key, const void *alpha, size_t bitWidthIn, size_t elementSize, size_t elementNum)
{
    const size_t rowBytes = ((size_t)1 << bitWidthIn) / 8;
    for (size_t i = 0; i < elementNum; i++)
    {
        uint64_t a = modbits(ld_el(alpha, i, elementSize), bitWidthIn);
        ((uint8_t *)key)[i * rowBytes + a / 8] ^= (uint8_t)(1u << (a % 8));
    }
}

/* otttLutEval: src/impl/ottt.h:26-192. E = number of set key bits; T_k = sum over set
 * bits i of lut[((x - i) mod 2^n) + k 2^n]; party 0 negates. */
void oracle_otttLutEval(void *sharedOutE, void *sharedOutT, const void *maskedX, const void *key, int partyId,
                        const void *lookUpTable, size_t lutNum, size_t bitWidthIn, size_t elementSize,
                        size_t elementNum)
{
    const size_t   es = elementSize, dom = (size_t)1 << bitWidthIn, mask = dom - 1;
    const uint64_t M  = esmask(es);
    ORACLE_PARALLEL_FOR
    for (long long ii = 0; ii < (long long)elementNum; ii++)
    {
        size_t         i   = (size_t)ii;
        const uint8_t *row = (const uint8_t *)key + i * (dom / 8);
        size_t         x   = (size_t)ld_el(maskedX, i, es);
        uint64_t       E   = 0;
        uint64_t      *T   = (uint64_t *)calloc(lutNum ? lutNum : 1, sizeof(uint64_t));
        for (size_t b = 0; b < dom; b++)
        {
            if (!((row[b >> 3] >> (b & 7)) & 1)) continue;
            E += 1;
            size_t idx = (x - b) & mask;
            for (size_t q = 0; q < lutNum; q++) T[q] += ld_el(lookUpTable, idx + q * dom, es);
        }
        if (partyId == 0)
        {
            E = 0 - E;
            for (size_t q = 0; q < lutNum; q++) T[q] = 0 - T[q];
        }
        st_el(sharedOutE, i, es, E & M);
        for (size_t q = 0; q < lutNum; q++) st_el(sharedOutT, i * lutNum + q, es, T[q] & M);
        free(T);
    }
}
