/* Test infrastructure: the CPU oracle.  A plain-C restatement of the reference
 * algorithm for the point-cloud neighbour-search path of
 * derivada/octrees-benchmark.  Every function names the reference file:line it
 * follows.  It is the checker for the CUDA path and never the thing measured
 * or shipped; only tests/, tests/golden/make_golden.py and bench.py's CPU
 * baseline load it.  It is pinned against the compiled reference
 * (oracle/_ref) and the golden fixtures under tests/golden/.
 *
 * Build: make -C oracle port   (gcc -O2 -ffp-contract=off: no FMA contraction,
 * like the reference's release flags, which carry no -mfma). */
#include "octree_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXD 21u
#define UPPER (1ull << 63)
#define MAXC ((1ull << MAXD) - 1ull)

enum { OUTSIDE = 0, OVERLAP = 1, INSIDE = 2 };

static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

/* ---- key algebra: inc/encoding/point_encoder.hpp:562-645 ---- */
static inline uint32_t key_level(uint64_t range) {          /* getLevel 568-573 */
    if (range == UPPER) return 0;
    return (uint32_t)(clz64(range - 1) - 1) / 3u;
}
static inline uint32_t key_sibling(uint64_t code, uint32_t level) { /* getSiblingId 576-579 */
    return (uint32_t)((code >> (3u * (MAXD - level))) & 7u);
}
static inline uint64_t key_node_range(uint32_t level) {     /* nodeRange 591-597 */
    return 1ull << (3u * (MAXD - level));
}
static inline uint64_t key_placeholder(uint64_t code, uint32_t level) { /* encodePlaceholderBit 613-618 */
    uint64_t ret = (level == 0) ? (code >> 63) : (code >> (3u * (MAXD - level)));
    return (1ull << (3u * level)) | ret;
}
static inline uint32_t key_prefix_len(uint64_t code) {      /* decodePrefixLength 600-602 */
    return (uint32_t)(63 - clz64(code));
}
static inline uint64_t key_unplaceholder(uint64_t code) {   /* decodePlaceholderBit 621-627 */
    uint32_t pl = key_prefix_len(code);
    uint64_t ret = code ^ (1ull << pl);
    return ret << (3u * MAXD - pl);
}
static inline int32_t key_common_prefix(uint64_t a, uint64_t b) { /* commonPrefix 630-632 */
    return (int32_t)clz64(a ^ b) - 1;
}
static inline uint32_t key_octal_digit(uint64_t code, uint32_t pos) { /* octalDigit 635-637 */
    return (uint32_t)((code >> (3u * (MAXD - pos))) & 7u);
}
static inline uint32_t key_log8ceil(uint64_t n) {           /* log8ceil 640-645 */
    if (n == 0) return 0;
    int lz = clz64(n - 1);
    return MAXD - (uint32_t)(lz - 1) / 3u;
}

/* ---- bounding box: mbb (inc/geometry/box.hpp:95-137), Box(pair) (18-21),
 *      then Box(center, radii) (17) as PointEncoder::sortPoints does
 *      (point_encoder.hpp:490-494) ---- */
void orc_bbox(const double* xyz, uint64_t n, double* box) {
    double mn[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    double mx[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    for (uint64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            double v = xyz[3 * i + a];
            mn[a] = (v < mn[a]) ? v : mn[a]; /* std::min(a, b) = (b < a) ? b : a */
            mx[a] = (mx[a] < v) ? v : mx[a]; /* std::max(a, b) = (a < b) ? b : a */
        }
    for (int a = 0; a < 3; ++a) {
        double r = (mx[a] - mn[a]) / 2.0;            /* radii = (max - min) / 2 */
        double c = mn[a] + (mx[a] - mn[a]) / 2.0;    /* midpoint (util.hpp:140) */
        box[a] = c;
        box[3 + a] = r;
        box[6 + a] = c - r;                          /* Box(center, radii): min = c - r */
        box[9 + a] = c + r;                          /*                     max = c + r */
    }
}

/* double -> uint_fast32_t (64-bit) conversion as x86-64 code does it: values
 * below 2^63 (and NaN, which compares unordered) go through the signed
 * truncation, whose out-of-range result is 0x8000000000000000; values from 2^63
 * up go through (v - 2^63) and an xor of the top bit. */
static uint64_t x86_cvt_u64(double v) {
    if (v != v) return 1ull << 63;
    if (v < 9223372036854775808.0) {
        if (v <= -9223372036854775808.0) return 1ull << 63;
        return (uint64_t)(int64_t)v;
    }
    double w = v - 9223372036854775808.0;
    uint64_t s = (w < 9223372036854775808.0) ? (uint64_t)(int64_t)w : (1ull << 63);
    return s ^ (1ull << 63);
}

/* PointEncoder::getAnchorCoords, one axis (point_encoder.hpp:37-49) */
uint64_t orc_anchor(double p, double c, double r) {
    double t = ((p - c) + r) / (2 * r);
    uint64_t u = x86_cvt_u64(t * (double)(1 << MAXD));
    return u < MAXC ? u : MAXC;
}

/* Morton: libmorton m3D_e_BMI / m3D_d_BMI (libmorton/morton_BMI.h:40-58):
 * x goes to bit 3i, y to 3i+1, z to 3i+2. */
uint64_t orc_morton_encode(uint64_t x, uint64_t y, uint64_t z) {
    uint64_t k = 0;
    for (uint32_t i = 0; i < MAXD; ++i) {
        k |= ((x >> i) & 1ull) << (3 * i);
        k |= ((y >> i) & 1ull) << (3 * i + 1);
        k |= ((z >> i) & 1ull) << (3 * i + 2);
    }
    return k;
}
void orc_morton_decode(uint64_t key, uint64_t* x, uint64_t* y, uint64_t* z) {
    uint64_t a = 0, b = 0, c = 0;
    for (uint32_t i = 0; i < MAXD; ++i) {
        a |= ((key >> (3 * i)) & 1ull) << i;
        b |= ((key >> (3 * i + 1)) & 1ull) << i;
        c |= ((key >> (3 * i + 2)) & 1ull) << i;
    }
    *x = a; *y = b; *z = c;
}

/* Hilbert: HilbertEncoder3D::encode (inc/encoding/hilbert_encoder_3d.hpp:29-66) */
uint64_t orc_hilbert_encode(uint64_t x64, uint64_t y64, uint64_t z64) {
    static const uint32_t lut[8] = {0, 1, 3, 2, 7, 6, 4, 5};
    uint32_t x = (uint32_t)x64, y = (uint32_t)y64, z = (uint32_t)z64;
    uint64_t key = 0;
    for (int level = (int)MAXD - 1; level >= 0; --level) {
        uint32_t xi = (x >> level) & 1u, yi = (y >> level) & 1u, zi = (z >> level) & 1u;
        uint32_t oct = (xi << 2) | (yi << 1) | zi;
        key = (key << 3) | lut[oct];
        uint32_t nyi = !yi, nzi = !zi;
        x ^= 0u - (xi & (nyi | zi));
        y ^= 0u - ((xi & (yi | zi)) | (yi & nzi));
        z ^= 0u - ((xi & nyi & nzi) | (yi & nzi));
        if (zi) {               /* rotate x, y, z -> y, z, x */
            uint32_t t = x; x = y; y = z; z = t;
        } else if (!yi) {       /* swap x and z */
            uint32_t t = x; x = z; z = t;
        }
    }
    return key;
}

/* HilbertEncoder3D::decode (hilbert_encoder_3d.hpp:256-289) */
void orc_hilbert_decode(uint64_t code, uint64_t* ox, uint64_t* oy, uint64_t* oz) {
    uint64_t x = 0, y = 0, z = 0;
    for (uint32_t level = 0; level < MAXD; ++level) {
        uint64_t oct = (code >> (3 * level)) & 7u;
        uint64_t xi = oct >> 2, yi = (oct >> 1) & 1u, zi = oct & 1u;
        if (yi ^ zi) {          /* rotate x, y, z -> z, x, y */
            uint64_t t = x; x = z; z = y; y = t;
        } else if ((!xi && !yi && !zi) || (xi && yi && zi)) {
            uint64_t t = x; x = z; z = t;
        }
        uint64_t mask = (1ull << level) - 1ull;
        uint64_t nxi = !xi, nyi = !yi, nzi = !zi;
        x ^= mask & (0ull - (xi & (yi | zi)));
        y ^= mask & (0ull - ((xi & (nyi | nzi)) | (nxi & yi & zi)));
        z ^= mask & (0ull - ((xi & nyi & nzi) | (yi & zi)));
        x |= xi << level;
        y |= (xi ^ yi) << level;
        z |= (yi ^ zi) << level;
    }
    *ox = x; *oy = y; *oz = z;
}

static inline uint64_t sfc_encode(int enc, uint64_t x, uint64_t y, uint64_t z) {
    return enc == 5 ? orc_hilbert_encode(x, y, z) : orc_morton_encode(x, y, z);
}
static inline void sfc_decode(int enc, uint64_t k, uint64_t* x, uint64_t* y, uint64_t* z) {
    if (enc == 5) orc_hilbert_decode(k, x, y, z); else orc_morton_decode(k, x, y, z);
}

/* encodePoints -> encodeFromPoint (point_encoder.hpp:54-63, morton_encoder_3d.hpp:48-52) */
void orc_encode(int encoder, const double* xyz, uint64_t n, const double* box, uint64_t* keys) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        uint64_t c[3];
        for (int a = 0; a < 3; ++a) c[a] = orc_anchor(xyz[3 * i + a], box[a], box[3 + a]);
        keys[i] = sfc_encode(encoder, c[0], c[1], c[2]);
    }
}

/* sortPoints: 8 passes x 8-bit LSD radix sort, stable (point_encoder.hpp:285-383).
 * keys are sorted in place; perm[i] = input position of the i-th sorted key. */
void orc_sort(uint64_t* keys, uint64_t n, uint32_t* perm) {
    uint64_t* kb = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint32_t* pb = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    for (int pass = 0; pass < 8; ++pass) {
        int shift = pass * 8;
        uint64_t hist[256] = {0};
        for (uint64_t i = 0; i < n; ++i) hist[(keys[i] >> shift) & 255u]++;
        uint64_t off = 0;
        for (int b = 0; b < 256; ++b) { uint64_t v = hist[b]; hist[b] = off; off += v; }
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t pos = hist[(keys[i] >> shift) & 255u]++;
            kb[pos] = keys[i];
            pb[pos] = perm[i];
        }
        memcpy(keys, kb, sizeof(uint64_t) * n);
        memcpy(perm, pb, sizeof(uint32_t) * n);
    }
    free(kb);
    free(pb);
}

/* ---------------- linear octree (inc/structures/linear_octree.hpp) ---------------- */

struct orc_tree {
    int encoder;
    uint64_t n;
    uint32_t nLeaf, nInternal, nTotal, maxDepthSeen;
    uint32_t* offsets;   /* nTotal + 1 */
    uint64_t* ranges;    /* nTotal x (first, last) */
    double* centers;     /* nTotal x 3 */
    double radii[(MAXD + 1) * 3];
    double half[3];
};

typedef struct {
    uint64_t* leaves;  /* nleaf + 1 */
    uint64_t* counts;  /* nleaf */
    uint64_t nleaf;
} leaf_part;

static uint64_t lower_bound_u64(const uint64_t* a, uint64_t n, uint64_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}
static uint64_t upper_bound_u64(const uint64_t* a, uint64_t n, uint64_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (!(v < a[mid])) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* computeNodeCounts / calculateNodeCount (291-321) */
static void compute_node_counts(leaf_part* lp, const uint64_t* codes, uint64_t ncodes) {
    uint64_t n = lp->nleaf, first, last;
    if (ncodes > 0) {
        first = upper_bound_u64(lp->leaves, n + 1, codes[0]) - 1;
        last = upper_bound_u64(lp->leaves, n + 1, codes[ncodes - 1]);
    } else {
        first = n; last = n;
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (i < first || i >= last) lp->counts[i] = 0;
        else lp->counts[i] = lower_bound_u64(codes, ncodes, lp->leaves[i + 1]) -
                             lower_bound_u64(codes, ncodes, lp->leaves[i]);
    }
}

/* siblingAndLevel (206-222) */
static void sibling_and_level(const leaf_part* lp, uint64_t i, int32_t* sib, uint32_t* level) {
    uint64_t node = lp->leaves[i];
    uint64_t range = lp->leaves[i + 1] - node;
    uint32_t l = key_level(range);
    *level = l;
    if (l == 0) { *sib = -1; return; }
    uint32_t sid = key_sibling(node, l);
    int on = lp->leaves[i - sid + 8] == lp->leaves[i - sid] + key_node_range(l - 1);
    *sib = on ? (int32_t)sid : -1;
}

/* calculateNodeOp (173-196) */
static uint64_t node_op(const leaf_part* lp, uint64_t i, uint64_t max_leaf, uint32_t* max_depth) {
    int32_t sib; uint32_t level;
    sibling_and_level(lp, i, &sib, &level);
    if (sib > 0) {
        uint64_t p = i - (uint64_t)sib, s = 0;
        for (int c = 0; c < 8; ++c) s += lp->counts[p + c];
        if (s <= max_leaf) return 0;
    }
    uint32_t cnt = (uint32_t)lp->counts[i];
    if (cnt > max_leaf && level < MAXD) {
        if (*max_depth < level + 1) *max_depth = level + 1;
        return 8;
    }
    return 1;
}

/* buildOctreeLeaves / updateOctreeLeaves / rebalanceTree / processNode (232-283, 458-489) */
static void build_leaves(leaf_part* lp, const uint64_t* codes, uint64_t n, uint64_t max_leaf, uint32_t* max_depth) {
    lp->nleaf = 1;
    lp->leaves = (uint64_t*)malloc(2 * sizeof(uint64_t));
    lp->counts = (uint64_t*)malloc(sizeof(uint64_t));
    lp->leaves[0] = 0; lp->leaves[1] = UPPER;
    lp->counts[0] = n;
    for (;;) {
        uint64_t nl = lp->nleaf;
        uint64_t* ops = (uint64_t*)calloc(nl + 1, sizeof(uint64_t));
        int converged = 1;
        for (uint64_t i = 0; i < nl; ++i) {
            ops[i] = node_op(lp, i, max_leaf, max_depth);
            if (ops[i] != 1) converged = 0;
        }
        if (converged) { free(ops); break; }
        /* exclusive scan over nl + 1 entries (325-333) */
        uint64_t a = 0, b = 0;
        for (uint64_t i = 0; i <= nl; ++i) { a += ops[i]; ops[i] = b; b = a; }
        uint64_t nn = ops[nl];
        uint64_t* nleaves = (uint64_t*)malloc((nn + 1) * sizeof(uint64_t));
        nleaves[nn] = lp->leaves[nl];
        for (uint64_t i = 0; i < nl; ++i) {
            uint64_t op = ops[i + 1] - ops[i];
            if (op == 0) continue;
            uint64_t node = lp->leaves[i];
            uint32_t level = key_level(lp->leaves[i + 1] - node);
            uint64_t at = ops[i];
            nleaves[at] = node;
            if (op > 1) {
                uint32_t ld = key_log8ceil(op);
                uint64_t gap = key_node_range(level + ld);
                for (uint64_t s = 1; s < op; ++s) nleaves[at + s] = nleaves[at + s - 1] + gap;
            }
        }
        free(ops);
        free(lp->leaves);
        free(lp->counts);
        lp->leaves = nleaves;
        lp->nleaf = nn;
        lp->counts = (uint64_t*)malloc((nn ? nn : 1) * sizeof(uint64_t));
        compute_node_counts(lp, codes, n);
    }
}

/* binaryKeyWeight / digitWeight (336-350) */
static int32_t digit_weight(uint32_t d) {
    int32_t m = -(int32_t)(d >= 4);
    return ((int32_t)(7 - d) & m) - ((int32_t)d & ~m);
}
static int32_t binary_key_weight(uint64_t key, uint32_t level) {
    int32_t r = 0;
    for (uint32_t l = 1; l <= level + 1; ++l) r += digit_weight(key_octal_digit(key, l));
    return r;
}

typedef struct { uint64_t prefix; int64_t i2l; } pfx_pair;
static int cmp_pfx(const void* a, const void* b) {
    const pfx_pair* x = (const pfx_pair*)a;
    const pfx_pair* y = (const pfx_pair*)b;
    if (x->prefix < y->prefix) return -1;
    if (x->prefix > y->prefix) return 1;
    return (x->i2l < y->i2l) ? -1 : (x->i2l > y->i2l); /* prefixes are unique; keeps it stable anyway */
}

typedef struct {
    uint64_t* prefixes;
    int64_t* i2l;   /* internalToLeaf */
    int64_t* l2i;   /* leafToInternal */
    uint64_t level_range[MAXD + 2];
} inter_part;

/* computeInternalRanges (410-428), post-order recursion */
static void internal_ranges(orc_tree* t, const inter_part* ip, const uint64_t* layout, uint32_t node,
                            uint64_t* first, uint64_t* last) {
    if (t->offsets[node] == 0) {
        int64_t li = ip->i2l[node];
        t->ranges[2 * node] = layout[li];
        t->ranges[2 * node + 1] = layout[li + 1];
    } else {
        for (uint32_t o = 0; o < 8; ++o) {
            uint64_t f, l;
            uint32_t child = t->offsets[node] + o;
            internal_ranges(t, ip, layout, child, &f, &l);
            if (o == 0) t->ranges[2 * node] = f;
            else if (o == 7) t->ranges[2 * node + 1] = l;
        }
    }
    *first = t->ranges[2 * node];
    *last = t->ranges[2 * node + 1];
}

/* LinearOctree ctor -> buildOctree (567-605) */
orc_tree* orc_build(int encoder, const uint64_t* keys, uint64_t n, uint64_t max_leaf, const double* box) {
    orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
    t->encoder = encoder;
    t->n = n;
    /* setupBbox (439-455): halfLengths = 0.5f * eps * (max - min), eps = 1.0f / 2^21 */
    const double eps = (double)(1.0f / (float)(1 << MAXD));
    for (int a = 0; a < 3; ++a) t->half[a] = 0.5 * eps * (box[9 + a] - box[6 + a]);
    for (uint32_t l = 0; l <= MAXD; ++l)
        for (int a = 0; a < 3; ++a) t->radii[3 * l + a] = (double)(1ull << (MAXD - l)) * t->half[a];

    leaf_part lp;
    build_leaves(&lp, keys, n, max_leaf, &t->maxDepthSeen);
    uint64_t nLeaf = lp.nleaf;
    uint64_t* layout = (uint64_t*)malloc((nLeaf + 1) * sizeof(uint64_t));
    layout[0] = 0;
    for (uint64_t i = 0; i < nLeaf; ++i) layout[i + 1] = layout[i] + lp.counts[i];

    /* resize (491-503) */
    uint64_t nInternal = (nLeaf - 1) / 7, nTotal = nLeaf + nInternal;
    t->nLeaf = (uint32_t)nLeaf; t->nInternal = (uint32_t)nInternal; t->nTotal = (uint32_t)nTotal;
    t->offsets = (uint32_t*)calloc(nTotal + 1, sizeof(uint32_t));
    t->ranges = (uint64_t*)calloc(2 * nTotal, sizeof(uint64_t));
    t->centers = (double*)calloc(3 * nTotal, sizeof(double));
    inter_part ip;
    ip.prefixes = (uint64_t*)calloc(nTotal, sizeof(uint64_t));
    ip.i2l = (int64_t*)calloc(nTotal, sizeof(int64_t));
    ip.l2i = (int64_t*)calloc(nTotal, sizeof(int64_t));

    /* createUnsortedLayout (353-367) */
    for (uint64_t i = 0; i < nLeaf; ++i) {
        uint64_t key = lp.leaves[i];
        uint32_t level = key_level(lp.leaves[i + 1] - key);
        ip.prefixes[i + nInternal] = key_placeholder(key, level);
        ip.i2l[i + nInternal] = (int64_t)(i + nInternal);
        uint32_t plen = (uint32_t)key_common_prefix(key, lp.leaves[i + 1]);
        if (plen % 3 == 0 && i < nLeaf - 1) {
            int64_t oi = ((int64_t)i + binary_key_weight(key, plen / 3)) / 7;
            ip.prefixes[oi] = key_placeholder(key, plen / 3);
            ip.i2l[oi] = oi;
        }
    }
    /* buildOctreeInternal (510-548): sort (prefix, internalToLeaf) by prefix */
    pfx_pair* pairs = (pfx_pair*)malloc(nTotal * sizeof(pfx_pair));
    for (uint64_t i = 0; i < nTotal; ++i) { pairs[i].prefix = ip.prefixes[i]; pairs[i].i2l = ip.i2l[i]; }
    qsort(pairs, nTotal, sizeof(pfx_pair), cmp_pfx);
    for (uint64_t i = 0; i < nTotal; ++i) { ip.prefixes[i] = pairs[i].prefix; ip.i2l[i] = pairs[i].i2l; }
    free(pairs);
    for (uint64_t i = 0; i < nTotal; ++i) ip.l2i[ip.i2l[i]] = (int64_t)i;
    for (uint64_t i = 0; i < nTotal; ++i) ip.i2l[i] -= (int64_t)nInternal;
    /* getLevelRange (370-376) */
    for (uint32_t l = 0; l <= MAXD; ++l)
        ip.level_range[l] = lower_bound_u64(ip.prefixes, nTotal, key_placeholder(0, l));
    ip.level_range[MAXD + 1] = nTotal;
    /* linkTree (379-407) */
    for (uint64_t i = 0; i < nInternal; ++i) {
        int64_t a = ip.l2i[i];
        uint64_t prefix = ip.prefixes[a];
        uint64_t node_key = key_unplaceholder(prefix);
        uint32_t level = key_prefix_len(prefix) / 3;
        if (level >= MAXD) continue; /* the reference exits here; unreachable for valid input */
        uint64_t child_prefix = key_placeholder(node_key, level + 1);
        uint64_t s = ip.level_range[level + 1], e = ip.level_range[level + 2];
        uint64_t c = s + lower_bound_u64(ip.prefixes + s, e - s, child_prefix);
        if (c != e && ip.prefixes[c] == child_prefix) t->offsets[a] = (uint32_t)c;
    }
    uint64_t f, l;
    internal_ranges(t, &ip, layout, 0, &f, &l);
    /* computeGeometry (557-565) -> PointEncoder::getCenter (point_encoder.hpp:517-539) */
    const double* bmin = box + 6;
    for (uint64_t i = 0; i < nTotal; ++i) {
        uint64_t prefix = ip.prefixes[i];
        uint64_t start = key_unplaceholder(prefix);
        uint32_t level = key_prefix_len(prefix) / 3;
        uint64_t c[3];
        sfc_decode(encoder, start, &c[0], &c[1], &c[2]);
        uint64_t mask = ((1ull << MAXD) - 1) ^ ((1ull << (MAXD - level)) - 1);
        for (int a = 0; a < 3; ++a) {
            double lo = bmin[a] + (double)(c[a] & mask) * t->half[a] * 2;
            t->centers[3 * i + a] = lo + t->radii[3 * level + a];
        }
    }
    free(layout);
    free(lp.leaves);
    free(lp.counts);
    free(ip.prefixes);
    free(ip.i2l);
    free(ip.l2i);
    return t;
}

void orc_tree_info(const orc_tree* t, uint64_t* out) {
    out[0] = t->n; out[1] = t->nLeaf; out[2] = t->nInternal; out[3] = t->nTotal; out[4] = t->maxDepthSeen;
}

void orc_tree_arrays(const orc_tree* t, uint32_t* offsets, uint64_t* ranges, double* centers, double* radii,
                     double* half) {
    if (offsets) memcpy(offsets, t->offsets, (t->nTotal + 1) * sizeof(uint32_t));
    if (ranges) memcpy(ranges, t->ranges, 2 * t->nTotal * sizeof(uint64_t));
    if (centers) memcpy(centers, t->centers, 3 * t->nTotal * sizeof(double));
    if (radii) memcpy(radii, t->radii, sizeof(t->radii));
    if (half) memcpy(half, t->half, sizeof(t->half));
}

void orc_tree_free(orc_tree* t) {
    if (!t) return;
    free(t->offsets); free(t->ranges); free(t->centers); free(t);
}

/* ---------------- search kernels (inc/kernels/kernel_{2d,3d}.hpp) ---------------- */

typedef struct {
    int type;            /* 0 circle, 1 sphere, 2 square, 3 cube */
    double c[3], r, r2, bmin[3], bmax[3];
} kern;

static kern make_kernel(int type, const double* c, double r) {
    kern k;
    k.type = type;
    k.r = r;
    k.r2 = r * r;
    for (int a = 0; a < 3; ++a) { k.c[a] = c[a]; k.bmin[a] = c[a] - r; k.bmax[a] = c[a] + r; }
    return k;                                   /* KernelAbstract::makeBox (kernel_abstract.hpp:41-45) */
}

static inline double dmax0(double v) { return (v < 0.0) ? 0.0 : v; } /* std::max(v, 0.0) */

static int is_inside(const kern* k, const double* p) {
    switch (k->type) {
        case 1: { /* KernelSphere::isInside (kernel_3d.hpp:168-179), strict */
            double d1 = p[0] - k->c[0], d2 = p[1] - k->c[1], d3 = p[2] - k->c[2];
            return d1 * d1 + d2 * d2 + d3 * d3 < k->r2;
        }
        case 0: { /* KernelCircle::isInside (kernel_2d.hpp:53-63) */
            double d1 = p[0] - k->c[0], d2 = p[1] - k->c[1];
            return d1 * d1 + d2 * d2 <= k->r2;
        }
        case 3: /* KernelCube::isInside (kernel_3d.hpp:273-283), onInterval (util.hpp:134) */
            return p[0] >= k->bmin[0] && p[0] <= k->bmax[0] && p[1] >= k->bmin[1] && p[1] <= k->bmax[1] &&
                   p[2] >= k->bmin[2] && p[2] <= k->bmax[2];
        default: /* KernelSquare::isInside (kernel_2d.hpp:153-162) */
            return p[0] >= k->bmin[0] && p[0] <= k->bmax[0] && p[1] >= k->bmin[1] && p[1] <= k->bmax[1];
    }
}

/* boxIntersect(center, Vector radii) overloads: sphere kernel_3d.hpp:222-264,
 * cube 318-343, circle kernel_2d.hpp:107-144, square 195-218 */
static int box_intersect(const kern* k, const double* oc, const double* orr) {
    switch (k->type) {
        case 1: {
            double dx = fabs(k->c[0] - oc[0]), dy = fabs(k->c[1] - oc[1]), dz = fabs(k->c[2] - oc[2]);
            double rx = orr[0], ry = orr[1], rz = orr[2];
            if (dx > k->r + rx || dy > k->r + ry || dz > k->r + rz) return OUTSIDE;
            double cx = dx + rx, cy = dy + ry, cz = dz + rz;
            if (cx * cx + cy * cy + cz * cz <= k->r2) return INSIDE;
            int ni = (dx < rx) + (dy < ry) + (dz < rz);
            if (ni > 1) return OVERLAP;
            dx = dmax0(dx - rx); dy = dmax0(dy - ry); dz = dmax0(dz - rz);
            if (dx * dx + dy * dy + dz * dz <= k->r2) return OVERLAP;
            return OUTSIDE;
        }
        case 0: {
            double dx = fabs(k->c[0] - oc[0]), dy = fabs(k->c[1] - oc[1]);
            double rx = orr[0], ry = orr[1];
            if (dx > k->r + rx || dy > k->r + ry) return OUTSIDE;
            double cx = dx + rx, cy = dy + ry;
            if (cx * cx + cy * cy <= k->r2) return INSIDE;
            int ni = (dx < rx) + (dy < ry);
            if (ni > 1) return OVERLAP;
            dx = dmax0(dx - rx); dy = dmax0(dy - ry);
            if (dx * dx + dy * dy <= k->r2) return OVERLAP;
            return OUTSIDE;
        }
        case 3: {
            double hx = oc[0] + orr[0], lx = oc[0] - orr[0];
            double hy = oc[1] + orr[1], ly = oc[1] - orr[1];
            double hz = oc[2] + orr[2], lz = oc[2] - orr[2];
            if (hx < k->bmin[0] || hy < k->bmin[1] || hz < k->bmin[2] || lx > k->bmax[0] || ly > k->bmax[1] ||
                lz > k->bmax[2])
                return OUTSIDE;
            if (hx <= k->bmax[0] && hy <= k->bmax[1] && hz <= k->bmax[2] && lx >= k->bmin[0] && ly >= k->bmin[1] &&
                lz >= k->bmin[2])
                return INSIDE;
            return OVERLAP;
        }
        default: {
            double hx = oc[0] + orr[0], lx = oc[0] - orr[0];
            double hy = oc[1] + orr[1], ly = oc[1] - orr[1];
            if (hx < k->bmin[0] || hy < k->bmin[1] || lx > k->bmax[0] || ly > k->bmax[1]) return OUTSIDE;
            if (hx <= k->bmax[0] && hy <= k->bmax[1] && lx >= k->bmin[0] && ly >= k->bmin[1]) return INSIDE;
            return OVERLAP;
        }
    }
}

/* Kernel3D::boxOverlap / Kernel2D::boxOverlap, Vector overloads
 * (kernel_3d.hpp:141-156, kernel_2d.hpp:29-41) */
static int box_overlap(const kern* k, const double* oc, const double* orr) {
    int dims = (k->type == 1 || k->type == 3) ? 3 : 2;
    for (int a = 0; a < dims; ++a)
        if (oc[a] + orr[a] < k->bmin[a]) return 0;
    for (int a = 0; a < dims; ++a)
        if (oc[a] - orr[a] > k->bmax[a]) return 0;
    return 1;
}

/* ---------------- traversal + searches ---------------- */

typedef struct {
    uint64_t* out;       /* index output (NULL: count only) */
    uint64_t* pairs;     /* range output for neighborsStruct (NULL: count only) */
    uint64_t count;      /* indices emitted (or ranges, in range mode) */
    int range_mode;
    uint32_t cut;        /* neighborsApprox: precisionLevel (NO_CUT: neighborsStruct) */
    int upper;           /* neighborsApprox: upperBound */
} sink;
#define NO_CUT 0xffffffffu

static void emit_index(sink* s, uint64_t i) {
    if (s->out) s->out[s->count] = i;
    s->count++;
}
static void emit_range(sink* s, uint64_t f, uint64_t l) {
    if (s->range_mode) {
        if (f <= l) { /* NeighborSet::addRange (neighbor_set.hpp:84-90) */
            if (s->pairs) { s->pairs[2 * s->count] = f; s->pairs[2 * s->count + 1] = l; }
            s->count++;
        }
    } else {
        for (uint64_t i = f; i < l; ++i) emit_index(s, i);
    }
}

/* continuationCriterion of neighborsStruct/neighborsPrune (698-714, 749-769), of
 * neighbors (800-802) and of neighborsApprox (979-1000: below precisionLevel the
 * octant's range is added in upper-bound mode and the search is cut, before any
 * box test) */
static int criterion(const orc_tree* t, const kern* k, int algo, uint32_t node, uint32_t depth, sink* s) {
    const double* oc = t->centers + 3 * (uint64_t)node;
    const double* orr = t->radii + 3 * depth;
    if (algo == 3 && depth > s->cut) {
        if (s->upper) emit_range(s, t->ranges[2 * node], t->ranges[2 * node + 1]);
        return 0;
    }
    if (algo == 1) return box_overlap(k, oc, orr);
    int j = box_intersect(k, oc, orr);
    if (j == INSIDE) {
        emit_range(s, t->ranges[2 * node], t->ranges[2 * node + 1]);
        return 0;
    }
    return j == OVERLAP;
}

/* endpointAction: neighborsStruct 716-732 (maximal runs), neighborsPrune 771-780,
 * neighbors 804-813 */
static void leaf_action(const orc_tree* t, const double* xyz, const kern* k, int algo, uint32_t node, sink* s) {
    uint64_t b = t->ranges[2 * node], e = t->ranges[2 * node + 1];
    if (algo == 3 && s->range_mode) {
        uint64_t rs = b;
        for (uint64_t i = b; i < e; ++i) {
            if (!is_inside(k, xyz + 3 * i)) {
                if (rs < i) emit_range(s, rs, i);
                rs = i + 1;
            }
        }
        if (rs < e) emit_range(s, rs, e);
        return;
    }
    for (uint64_t i = b; i < e; ++i)
        if (is_inside(k, xyz + 3 * i)) emit_index(s, i);
}

/* singleTraversal (653-686) */
static void single_traversal(const orc_tree* t, const double* xyz, const kern* k, int algo, sink* s) {
    if (!criterion(t, k, algo, 0, 0, s)) return;
    if (t->offsets[0] == 0) { leaf_action(t, xyz, k, algo, 0, s); return; }
    uint32_t st_node[128], st_depth[128];
    st_node[0] = 0; st_depth[0] = 0;
    uint32_t sp = 1, node = 0, depth = 0;
    do {
        for (uint32_t o = 0; o < 8; ++o) {
            uint32_t child = t->offsets[node] + o;
            if (criterion(t, k, algo, child, depth + 1, s)) {
                if (t->offsets[child] == 0) leaf_action(t, xyz, k, algo, child, s);
                else if (sp < 128) { st_node[sp] = child; st_depth[sp] = depth + 1; ++sp; }
            }
        }
        --sp;
        node = st_node[sp];
        depth = st_depth[sp];
    } while (node != 0);
}

void orc_radius_count(const orc_tree* t, const double* xyz, int kernel, int algo, const double* centers,
                      uint64_t nq, const double* radii, uint64_t* counts) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        kern k = make_kernel(kernel, centers + 3 * q, radii[q]);
        sink s = {NULL, NULL, 0, 0, NO_CUT, 0};
        single_traversal(t, xyz, &k, algo, &s);
        counts[q] = s.count;
    }
}

void orc_radius_fill(const orc_tree* t, const double* xyz, int kernel, int algo, const double* centers,
                     uint64_t nq, const double* radii, const uint64_t* offsets, uint64_t* idx) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        kern k = make_kernel(kernel, centers + 3 * q, radii[q]);
        sink s = {idx + offsets[q], NULL, 0, 0, NO_CUT, 0};
        single_traversal(t, xyz, &k, algo, &s);
    }
}

void orc_approx_ranges_count(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                             uint64_t nq, const double* radii, uint32_t level, int upper, uint64_t* counts) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        kern k = make_kernel(kernel, centers + 3 * q, radii[q]);
        sink s = {NULL, NULL, 0, 1, level, upper};
        single_traversal(t, xyz, &k, 3, &s);
        counts[q] = s.count;
    }
}

void orc_approx_ranges_fill(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                            uint64_t nq, const double* radii, uint32_t level, int upper, const uint64_t* offsets,
                            uint64_t* pairs) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        kern k = make_kernel(kernel, centers + 3 * q, radii[q]);
        sink s = {NULL, pairs + 2 * offsets[q], 0, 1, level, upper};
        single_traversal(t, xyz, &k, 3, &s);
    }
}

void orc_struct_ranges_count(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                             uint64_t nq, const double* radii, uint64_t* counts) {
    orc_approx_ranges_count(t, xyz, kernel, centers, nq, radii, NO_CUT, 0, counts);
}

void orc_struct_ranges_fill(const orc_tree* t, const double* xyz, int kernel, const double* centers,
                            uint64_t nq, const double* radii, const uint64_t* offsets, uint64_t* pairs) {
    orc_approx_ranges_fill(t, xyz, kernel, centers, nq, radii, NO_CUT, 0, offsets, pairs);
}

/* ---------------- kNN: best-first search (linear_octree.hpp:819-942) ---------------- */

typedef struct { uint64_t index; uint32_t is_oct, depth; double d2; } heap_ent;
typedef struct { heap_ent* a; uint64_t n, cap; } minheap;

/* The reference orders heap entries by sqDist only (OctantPointIndex::operator<,
 * linear_octree.hpp:837-840), which leaves equal distances in unspecified order.
 * The oracle breaks those ties deterministically: octants before points (so
 * every octant that can hold a point at that distance is opened first), then
 * the lower index.  The points it returns at the k-th distance are therefore
 * the lowest-indexed of all points at exactly that distance. */
static inline int ent_less(const heap_ent* x, const heap_ent* y) {
    if (x->d2 < y->d2) return 1;
    if (y->d2 < x->d2) return 0;
    if (x->is_oct != y->is_oct) return x->is_oct > y->is_oct;
    return x->index < y->index;
}

static void heap_push(minheap* h, heap_ent e) {
    if (h->n == h->cap) {
        h->cap = h->cap ? 2 * h->cap : 512;
        h->a = (heap_ent*)realloc(h->a, h->cap * sizeof(heap_ent));
    }
    uint64_t i = h->n++;
    while (i > 0) {
        uint64_t p = (i - 1) / 2;
        if (!ent_less(&e, &h->a[p])) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = e;
}
static heap_ent heap_pop(minheap* h) {
    heap_ent top = h->a[0];
    heap_ent last = h->a[--h->n];
    uint64_t i = 0;
    for (;;) {
        uint64_t l = 2 * i + 1, r = l + 1, m = i;
        const heap_ent* mm = &last;
        if (l < h->n && ent_less(&h->a[l], mm)) { m = l; mm = &h->a[l]; }
        if (r < h->n && ent_less(&h->a[r], mm)) { m = r; }
        if (m == i) break;
        h->a[i] = h->a[m];
        i = m;
    }
    if (h->n) h->a[i] = last;
    return top;
}

/* distPointsSquared (844-851) */
static inline double dist_pp(const double* p, const double* q) {
    double dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    return dx * dx + dy * dy + dz * dz;
}
/* distPointOctantSquared (854-878) */
static inline double dist_po(const double* p, const double* oc, const double* orr) {
    double d[3];
    for (int a = 0; a < 3; ++a) {
        double lo = oc[a] - orr[a], hi = oc[a] + orr[a];
        double m = (hi < p[a]) ? hi : p[a];      /* std::min(p, hi) */
        double c = (lo < m) ? m : lo;            /* std::max(lo, m) */
        d[a] = p[a] - c;
    }
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
}

void orc_knn(const orc_tree* t, const double* xyz, uint64_t n, const double* centers, uint64_t nq, uint64_t k,
             uint64_t* idx, double* d2, uint64_t* counts) {
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        const double* p = centers + 3 * q;
        minheap h = {NULL, 0, 0};
        heap_ent root = {0, 1, 0, 0.0};
        heap_push(&h, root);
        uint64_t got = 0, want = n < k ? n : k;
        while (got < want && h.n > 0) {
            heap_ent top = heap_pop(&h);
            if (top.is_oct) {
                uint32_t node = (uint32_t)top.index;
                if (t->offsets[node] == 0) {
                    for (uint64_t i = t->ranges[2 * node]; i < t->ranges[2 * node + 1]; ++i) {
                        heap_ent e = {i, 0, 0, dist_pp(p, xyz + 3 * i)};
                        heap_push(&h, e);
                    }
                } else {
                    uint32_t cd = top.depth + 1;
                    for (uint32_t o = 0; o < 8; ++o) {
                        uint32_t c = t->offsets[node] + o;
                        heap_ent e = {c, 1, cd, dist_po(p, t->centers + 3 * (uint64_t)c, t->radii + 3 * cd)};
                        heap_push(&h, e);
                    }
                }
            } else {
                idx[q * k + got] = top.index;
                d2[q * k + got] = top.d2;
                ++got;
            }
        }
        for (uint64_t j = got; j < k; ++j) { idx[q * k + j] = UINT64_MAX; d2[q * k + j] = INFINITY; }
        counts[q] = got;
        free(h.a);
    }
}
