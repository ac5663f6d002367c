/*
 * ORACLE - test infrastructure only.  A plain-C CPU restatement of the
 * reference's spectral placement hot path, used by tests/, the smoke check
 * and the CPU-baseline leg of bench.py as the checker.  The product never
 * links or calls it.
 *
 * Pinned against: the reference's own golden vectors
 * (tests/native/integer_correlation_tests.cpp:11-60,
 * engine/pack_compute/tests/correlation_tests.cpp:292-481) and the reference
 * C++ compiled here (oracle/_ref/libspk_ref.so, built by oracle/ref/Makefile).
 *
 * Functions and the reference code each restates:
 *   oracle_correlate_int       tests/support/src/integer_correlation.cpp:127-181
 *   oracle_correlate_binary    engine/pack_compute/src/correlation.cpp:238-592 (exact result)
 *   oracle_correlate_proximity correlation.cpp:238-592, proximity variant (exact result,
 *                              correctly rounded)
 *   oracle_build_proximity     engine/pack_solver/src/field_proximity.hpp:32-132
 *   oracle_fsum                correctly rounded sum (Shewchuk expansions)
 *   oracle_broad_phase         engine/pack_geometry/src/validation.cpp:404-418 pair order with
 *                              separated_conservative_bounds, validation_kernel.cpp:1245-1261
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Correctly rounded sum of n doubles: Shewchuk's non-overlapping expansion
 * with the final round-half-even correction used by Python's math.fsum. */
double oracle_fsum(const double* values, int64_t n)
{
    double partials_fixed[64];
    double* partials = partials_fixed;
    int64_t count = 0, capacity = 64;
    for (int64_t k = 0; k < n; ++k) {
        double x = values[k];
        int64_t i = 0;
        for (int64_t j = 0; j < count; ++j) {
            double y = partials[j];
            if (fabs(x) < fabs(y)) {
                double t = x;
                x = y;
                y = t;
            }
            const double hi = x + y;
            const double lo = y - (hi - x);
            if (lo != 0.0) {
                partials[i++] = lo;
            }
            x = hi;
        }
        if (i >= capacity) {
            double* grown = (double*)malloc(sizeof(double) * (size_t)capacity * 2);
            memcpy(grown, partials, sizeof(double) * (size_t)i);
            if (partials != partials_fixed) {
                free(partials);
            }
            partials = grown;
            capacity *= 2;
        }
        partials[i++] = x;
        count = i;
    }
    double hi = 0.0;
    if (count > 0) {
        int64_t j = count - 1;
        hi = partials[j];
        double lo = 0.0;
        while (j > 0) {
            const double x = hi;
            const double y = partials[--j];
            hi = x + y;
            const double yr = hi - x;
            lo = y - yr;
            if (lo != 0.0) {
                break;
            }
        }
        if (j > 0 && ((lo < 0.0 && partials[j - 1] < 0.0) || (lo > 0.0 && partials[j - 1] > 0.0))) {
            const double y = lo * 2.0;
            const double x = hi + y;
            const double yr = x - hi;
            if (y == yr) {
                hi = x;
            }
        }
    }
    if (partials != partials_fixed) {
        free(partials);
    }
    return hi;
}

/* Direct integer full-range correlation with the test_support convention:
 * out(t) = sum_k B[t + origin + k] * K[k], t over every translation where the
 * kernel box meets the field box.  range_first receives the first translation
 * and out_shape the output extents.  Returns 0, or 1 on overflow. */
int oracle_correlate_int(const int64_t* blocked, const int64_t* bshape, const int64_t* kernel,
                         const int64_t* kshape, const int64_t* origin, int64_t* out, int64_t* range_first,
                         int64_t* out_shape)
{
    for (int a = 0; a < 3; ++a) {
        range_first[a] = -origin[a] - (kshape[a] - 1);
        out_shape[a] = bshape[a] + kshape[a] - 1;
    }
    for (int64_t tz = 0; tz < out_shape[2]; ++tz) {
        for (int64_t ty = 0; ty < out_shape[1]; ++ty) {
            for (int64_t tx = 0; tx < out_shape[0]; ++tx) {
                const int64_t t[3] = { tx + range_first[0], ty + range_first[1], tz + range_first[2] };
                int64_t sum = 0;
                for (int64_t kz = 0; kz < kshape[2]; ++kz) {
                    for (int64_t ky = 0; ky < kshape[1]; ++ky) {
                        for (int64_t kx = 0; kx < kshape[0]; ++kx) {
                            const int64_t bx = t[0] + origin[0] + kx, by = t[1] + origin[1] + ky,
                                          bz = t[2] + origin[2] + kz;
                            if (bx < 0 || by < 0 || bz < 0 || bx >= bshape[0] || by >= bshape[1] || bz >= bshape[2]) {
                                continue;
                            }
                            const int64_t term =
                                blocked[bx + bshape[0] * (by + bshape[1] * bz)] * kernel[kx + kshape[0] * (ky + kshape[1] * kz)];
                            if ((term > 0 && sum > INT64_MAX - term) || (term < 0 && sum < INT64_MIN - term)) {
                                return 1;
                            }
                            sum += term;
                        }
                    }
                }
                out[tx + out_shape[0] * (ty + out_shape[1] * tz)] = sum;
            }
        }
    }
    return 0;
}

/* CorrelationSpec convention (correlation.hpp:20-27): kernel cell i sits at
 * world translation + kernel_first + i, environment cell 0 at env_first.
 * Output covers E+K-1 per axis from t_first = env_first - kernel_first - (K-1).
 * Binary: exact integer overlap counts as doubles. */
void oracle_correlate_binary(const uint32_t* es, const uint32_t* ks, const int64_t* ef, const int64_t* kf,
                             const uint8_t* env, const uint8_t* ker, double* out, int64_t* t_first,
                             uint32_t* out_shape)
{
    uint32_t os[3];
    for (int a = 0; a < 3; ++a) {
        os[a] = es[a] + ks[a] - 1;
        out_shape[a] = os[a];
        t_first[a] = ef[a] - kf[a] - ((int64_t)ks[a] - 1);
    }
    for (uint32_t z = 0; z < os[2]; ++z) {
        for (uint32_t y = 0; y < os[1]; ++y) {
            for (uint32_t x = 0; x < os[0]; ++x) {
                const int64_t sx = (int64_t)x - (ks[0] - 1), sy = (int64_t)y - (ks[1] - 1), sz = (int64_t)z - (ks[2] - 1);
                uint64_t sum = 0;
                for (uint32_t kz = 0; kz < ks[2]; ++kz) {
                    const int64_t cz = kz + sz;
                    if (cz < 0 || cz >= es[2]) {
                        continue;
                    }
                    for (uint32_t ky = 0; ky < ks[1]; ++ky) {
                        const int64_t cy = ky + sy;
                        if (cy < 0 || cy >= es[1]) {
                            continue;
                        }
                        for (uint32_t kx = 0; kx < ks[0]; ++kx) {
                            const int64_t cx = kx + sx;
                            if (cx < 0 || cx >= es[0]) {
                                continue;
                            }
                            sum += (uint64_t)env[cx + (int64_t)es[0] * (cy + (int64_t)es[1] * cz)] *
                                   ker[kx + (int64_t)ks[0] * (ky + (int64_t)ks[1] * kz)];
                        }
                    }
                }
                out[x + (int64_t)os[0] * (y + (int64_t)os[1] * z)] = (double)sum;
            }
        }
    }
}

/* Proximity variant: the exact sum of the selected environment values,
 * correctly rounded to binary64. */
void oracle_correlate_proximity(const uint32_t* es, const uint32_t* ks, const int64_t* ef, const int64_t* kf,
                                const double* env, const uint8_t* ker, double* out, int64_t* t_first,
                                uint32_t* out_shape)
{
    uint32_t os[3];
    for (int a = 0; a < 3; ++a) {
        os[a] = es[a] + ks[a] - 1;
        out_shape[a] = os[a];
        t_first[a] = ef[a] - kf[a] - ((int64_t)ks[a] - 1);
    }
    const int64_t kn = (int64_t)ks[0] * ks[1] * ks[2];
    double* terms = (double*)malloc(sizeof(double) * (size_t)(kn ? kn : 1));
    for (uint32_t z = 0; z < os[2]; ++z) {
        for (uint32_t y = 0; y < os[1]; ++y) {
            for (uint32_t x = 0; x < os[0]; ++x) {
                const int64_t sx = (int64_t)x - (ks[0] - 1), sy = (int64_t)y - (ks[1] - 1), sz = (int64_t)z - (ks[2] - 1);
                int64_t n = 0;
                for (uint32_t kz = 0; kz < ks[2]; ++kz) {
                    const int64_t cz = kz + sz;
                    if (cz < 0 || cz >= es[2]) {
                        continue;
                    }
                    for (uint32_t ky = 0; ky < ks[1]; ++ky) {
                        const int64_t cy = ky + sy;
                        if (cy < 0 || cy >= es[1]) {
                            continue;
                        }
                        for (uint32_t kx = 0; kx < ks[0]; ++kx) {
                            const int64_t cx = kx + sx;
                            if (cx < 0 || cx >= es[0] || !ker[kx + (int64_t)ks[0] * (ky + (int64_t)ks[1] * kz)]) {
                                continue;
                            }
                            terms[n++] = env[cx + (int64_t)es[0] * (cy + (int64_t)es[1] * cz)];
                        }
                    }
                }
                out[x + (int64_t)os[0] * (y + (int64_t)os[1] * z)] = oracle_fsum(terms, n);
            }
        }
    }
    free(terms);
}

/* Exact squared EDT by separable lower envelopes, then exp(-sqrt(d2)/2);
 * 0 where no cell is occupied (field_proximity.hpp:32-132).  d2 (optional)
 * receives the squared distances, -1 for "no occupied cell".  Returns 0. */
int oracle_build_proximity(const uint32_t* shape, const uint8_t* occupied, double* values, int64_t* d2_out)
{
    const int64_t n = (int64_t)shape[0] * shape[1] * shape[2];
    const double inf = INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        values[i] = occupied[i] ? 0.0 : inf;
    }
    uint32_t longest = shape[0];
    if (shape[1] > longest) longest = shape[1];
    if (shape[2] > longest) longest = shape[2];
    double* line = (double*)malloc(sizeof(double) * longest);
    uint32_t* site_q = (uint32_t*)malloc(sizeof(uint32_t) * longest);
    int64_t* site_start = (int64_t*)malloc(sizeof(int64_t) * longest);
    const int64_t strides[3] = { 1, shape[0], (int64_t)shape[0] * shape[1] };
    for (int axis = 0; axis < 3; ++axis) {
        const uint32_t length = shape[axis];
        const int64_t stride = strides[axis];
        for (int64_t base = 0; base < n; ++base) {
            if ((base / stride) % length != 0) {
                continue;
            }
            int64_t count = 0;
            for (uint32_t q = 0; q < length; ++q) {
                line[q] = values[base + q * stride];
            }
            for (uint32_t q = 0; q < length; ++q) {
                if (!isfinite(line[q])) {
                    continue;
                }
                int64_t start = INT64_MIN;
                while (count > 0) {
                    const int64_t p = site_q[count - 1];
                    const int64_t numerator = (int64_t)line[q] - (int64_t)line[p] + (int64_t)q * q - p * p;
                    const int64_t denominator = 2 * ((int64_t)q - p);
                    start = numerator / denominator + (numerator % denominator < 0 ? -1 : 0) + 1;
                    if (start > site_start[count - 1]) {
                        break;
                    }
                    --count;
                }
                if (count == 0) {
                    start = INT64_MIN;
                }
                site_q[count] = q;
                site_start[count] = start;
                ++count;
            }
            int64_t site = 0;
            for (uint32_t q = 0; q < length; ++q) {
                while (site + 1 < count && site_start[site + 1] <= q) {
                    ++site;
                }
                if (count == 0) {
                    values[base + q * stride] = inf;
                }
                else {
                    const int64_t delta = (int64_t)q - site_q[site];
                    values[base + q * stride] = line[site_q[site]] + (double)(delta * delta);
                }
            }
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        if (d2_out) {
            d2_out[i] = isfinite(values[i]) ? (int64_t)values[i] : -1;
        }
        values[i] = isfinite(values[i]) ? exp(-sqrt(values[i]) / 2.) : 0.;
    }
    free(line);
    free(site_q);
    free(site_start);
    return 0;
}

/* ---- spectral page (engine/pack_solver/src/spectral_pipeline.cpp:1618-1857) ----
 * For every legal translation t = (env_first - kernel_first) + s,
 * 0 <= s <= E - K: overlap = exact u8 overlap count; ordinary pages keep
 * overlap == 0; score = .65 * top - .35 * prox / occ with prox the correctly
 * rounded exact sum of the proximity values under the kernel's ones and
 * top = (origin_z + pitch * t_z + max_z - c_min_z) / H; order by
 * (score, orientation, z, y, x); keep 32 entries strictly after the cursor.
 * A naive FP64 sum (error < 1e-7 here) screens candidates; every candidate
 * within 1e-6 of the page boundary is rescored with oracle_fsum. */
typedef struct {
    int64_t t[3];
    double score;
    int32_t direct_zero;
    int32_t reserved;
    uint64_t orientation;
    double binary_overlap;
} OracleCandidate;

static int oracle_rank_less(const OracleCandidate* l, const OracleCandidate* r)
{
    if (l->score != r->score) return l->score < r->score;
    if (l->orientation != r->orientation) return l->orientation < r->orientation;
    if (l->t[2] != r->t[2]) return l->t[2] < r->t[2];
    if (l->t[1] != r->t[1]) return l->t[1] < r->t[1];
    return l->t[0] < r->t[0];
}

static int cmp_candidates(const void* a, const void* b)
{
    const OracleCandidate* l = (const OracleCandidate*)a;
    const OracleCandidate* r = (const OracleCandidate*)b;
    return oracle_rank_less(l, r) ? -1 : oracle_rank_less(r, l) ? 1 : 0;
}

static double oracle_score(double p, uint64_t occ, int64_t tz, const double* lat, double max_z, double cmin_z,
                           double height)
{
    const double mean = p / (double)occ;
    const double world_z = lat[2] + lat[3] * (double)tz;
    const double top = (world_z + max_z - cmin_z) / height;
    return .65 * top - .35 * mean;
}

/* lat = {origin x, y, z, pitch}; returns the number of page entries (<= 32),
 * or -1 for an empty kernel. */
int oracle_page(const int64_t* env_first, const uint32_t* es, const uint8_t* occ, const double* prox,
                const int64_t* ker_first, const uint32_t* ks, const uint8_t* ker, const double* lat, double max_z,
                double cmin_z, double height, uint64_t orientation, const OracleCandidate* cursor,
                OracleCandidate* page)
{
    int64_t nk = 0;
    const int64_t kn = (int64_t)ks[0] * ks[1] * ks[2];
    int64_t* ones = (int64_t*)malloc(sizeof(int64_t) * (size_t)(kn ? kn : 1));
    for (uint32_t z = 0; z < ks[2]; ++z)
        for (uint32_t y = 0; y < ks[1]; ++y)
            for (uint32_t x = 0; x < ks[0]; ++x)
                if (ker[x + (int64_t)ks[0] * (y + (int64_t)ks[1] * z)])
                    ones[nk++] = x + (int64_t)es[0] * (y + (int64_t)es[1] * z);
    if (nk == 0) {
        free(ones);
        return -1;
    }
    for (int a = 0; a < 3; ++a) {
        if (es[a] < ks[a]) {
            free(ones);
            return 0;
        }
    }
    const int64_t legal[3] = { es[0] - ks[0] + 1, es[1] - ks[1] + 1, es[2] - ks[2] + 1 };
    const int64_t first[3] = { env_first[0] - ker_first[0], env_first[1] - ker_first[1], env_first[2] - ker_first[2] };
    const double band = 1e-6;
    /* screening list: every feasible candidate with its naive score */
    int64_t cap = 1024, n = 0;
    OracleCandidate* list = (OracleCandidate*)malloc(sizeof(OracleCandidate) * (size_t)cap);
    double* terms = (double*)malloc(sizeof(double) * (size_t)nk);
    for (int64_t sz = 0; sz < legal[2]; ++sz)
        for (int64_t sy = 0; sy < legal[1]; ++sy)
            for (int64_t sx = 0; sx < legal[0]; ++sx) {
                const int64_t base = sx + (int64_t)es[0] * (sy + (int64_t)es[1] * sz);
                int hit = 0;
                double naive = 0.0;
                for (int64_t i = 0; i < nk; ++i) {
                    if (occ[base + ones[i]]) {
                        hit = 1;
                        break;
                    }
                    naive += prox[base + ones[i]];
                }
                if (hit) continue;
                OracleCandidate c;
                c.t[0] = first[0] + sx;
                c.t[1] = first[1] + sy;
                c.t[2] = first[2] + sz;
                c.score = oracle_score(naive, (uint64_t)nk, c.t[2], lat, max_z, cmin_z, height);
                c.direct_zero = 1;
                c.reserved = 0;
                c.orientation = orientation;
                c.binary_overlap = 0.0;
                /* drop candidates certainly at or before the cursor */
                if (cursor && c.score < cursor->score - band) continue;
                if (n == cap) {
                    cap *= 2;
                    list = (OracleCandidate*)realloc(list, sizeof(OracleCandidate) * (size_t)cap);
                }
                list[n++] = c;
            }
    qsort(list, (size_t)n, sizeof(OracleCandidate), cmp_candidates);
    /* Walk in naive order, rescoring exactly, until 32 entries follow the
     * cursor and the next naive score is beyond the 32nd exact one + band. */
    OracleCandidate* kept = (OracleCandidate*)malloc(sizeof(OracleCandidate) * (size_t)(n ? n : 1));
    int64_t m = 0;
    double worst = INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        if (m >= 32 && list[i].score > worst + 2 * band) break;
        OracleCandidate c = list[i];
        const int64_t sx = c.t[0] - first[0], sy = c.t[1] - first[1], sz = c.t[2] - first[2];
        const int64_t base = sx + (int64_t)es[0] * (sy + (int64_t)es[1] * sz);
        for (int64_t k = 0; k < nk; ++k) terms[k] = prox[base + ones[k]];
        c.score = oracle_score(oracle_fsum(terms, nk), (uint64_t)nk, c.t[2], lat, max_z, cmin_z, height);
        if (cursor && !oracle_rank_less(cursor, &c)) continue;
        kept[m++] = c;
        if (m >= 32) {
            qsort(kept, (size_t)m, sizeof(OracleCandidate), cmp_candidates);
            worst = kept[31].score;
        }
    }
    qsort(kept, (size_t)m, sizeof(OracleCandidate), cmp_candidates);
    free(list);
    list = kept;
    const int count = (int)(m < 32 ? m : 32);
    for (int i = 0; i < count; ++i) page[i] = list[i];
    free(list);
    free(terms);
    free(ones);
    return count;
}

/* ---- validator broad phase (validation.cpp:404-418) ----
 * The validator's pair loop visits (first, second) for first = 0..n-1 and
 * second = 0..first-1, skipping pairs whose poses are both proven.  A pair
 * is certified disjoint by its posed conservative bounds when, on some axis,
 * nextafter(max + clearance, +inf) of one copy lies below the other copy's
 * min (validation_kernel.cpp:1252-1258); copies whose bounds are not finite
 * certify nothing.  Writes the uncertified pairs in visiting order as
 * (first, second) uint32 pairs, up to `capacity`, and returns their count. */
static int oracle_separated(const double* lo, const double* hi, const uint8_t* finite, int64_t i, int64_t j,
                            double clearance)
{
    if (!finite[i] || !finite[j]) return 0;
    for (int a = 0; a < 3; ++a) {
        const double x = nextafter(hi[3 * i + a] + clearance, INFINITY);
        const double y = nextafter(hi[3 * j + a] + clearance, INFINITY);
        if (x < lo[3 * j + a] || y < lo[3 * i + a]) return 1;
    }
    return 0;
}

int64_t oracle_broad_phase(const double* lo, const double* hi, const uint8_t* finite, const uint8_t* proven,
                           int64_t n, double clearance, uint32_t* pairs, int64_t capacity)
{
    int64_t count = 0;
    for (int64_t first = 0; first < n; ++first) {
        for (int64_t second = 0; second < first; ++second) {
            if (proven && proven[first] && proven[second]) continue;
            if (oracle_separated(lo, hi, finite, first, second, clearance)) continue;
            if (count < capacity) {
                pairs[2 * count] = (uint32_t)first;
                pairs[2 * count + 1] = (uint32_t)second;
            }
            ++count;
        }
    }
    return count;
}
