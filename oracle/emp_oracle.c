/*
 * CPU oracle for edge_matching_puzzle_b200 -- TEST INFRASTRUCTURE ONLY.
 * See emp_oracle.h for what it restates and how it is pinned.  Every
 * function below names the reference lines (relative to the reference
 * project root) whose behaviour it reproduces.
 */
#include "emp_oracle.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { K_CENTER = 0, K_BORDER = 1, K_CORNER = 2 };
enum { SIM_NONE = 0, SIM_HALF = 1, SIM_SIMILAR = 2 };

#define OP_MAXN 256

struct op_puzzle {
    uint32_t w, h, n;
    uint32_t col[OP_MAXN][4];
    uint8_t kind[OP_MAXN];
    uint8_t sim[OP_MAXN];
    uint32_t kind_index[OP_MAXN];
    uint32_t nb_kind[3];
    uint32_t members[3][OP_MAXN];
    uint32_t max_color, border_id, cs, max_code, id_size, dumped_id_size;
    uint32_t kind_bits[3], kind_words[3];
    uint32_t *binary[3];       /* [4*nb_kind]                            */
    uint64_t *idmask[3];       /* [4*nb_kind][kind_words]                */
    uint8_t twins[OP_MAXN][OP_MAXN / 8];
    int has_identical;
    int id_out_of_range;
    /* constraint table, emp_piece_db.h:770-827 */
    uint32_t *table_off;       /* [max_code+1] word offset or UINT32_MAX */
    uint8_t *table_kind;       /* [max_code+1]                           */
    uint64_t *table_pool;
    uint64_t table_words;
};

/* ------------------------------------------------------------------ */
/* bit helpers (quicky_bitfield<uint64_t>: bit i in word i/64, LSB first) */
static inline int bf_get(const uint64_t *w, uint32_t i) { return (int)((w[i >> 6] >> (i & 63)) & 1u); }
static inline void bf_set1(uint64_t *w, uint32_t i) { w[i >> 6] |= (uint64_t)1 << (i & 63); }
static inline void bf_clr(uint64_t *w, uint32_t i) { w[i >> 6] &= ~((uint64_t)1 << (i & 63)); }
static inline uint32_t bf_ffs(const uint64_t *w, uint32_t nwords)
{
    for (uint32_t i = 0; i < nwords; ++i)
        if (w[i]) return i * 64 + (uint32_t)__builtin_ctzll(w[i]) + 1;
    return 0;
}

static uint32_t nb_bits(uint32_t v) /* emp_piece_db.h:1529-1539 */
{
    uint32_t n = 0;
    while (v) { ++n; v >>= 1; }
    return n;
}

/* emp_piece.h:144-157 */
static uint8_t auto_similarity(const uint32_t *c)
{
    if (c[0] == c[2] && c[1] == c[3]) return c[0] == c[1] ? SIM_SIMILAR : SIM_HALF;
    return SIM_NONE;
}

/* emp_piece.h:208-220: this=a, p_piece=b, orientation o.  The reference
 * steps through a's sides by 2^similarity(a); the out-of-range read it does
 * once the index passes WEST cannot change the result (it returns true
 * either way), so it is not reproduced. */
static int compare_to(const op_puzzle *p, uint32_t a, uint32_t b, uint32_t o)
{
    if (a == b) return 1;
    uint32_t inc = 1u << p->sim[a];
    uint32_t idx = 0;
    while (idx <= 3 && p->col[a][idx] == p->col[b][(idx + o) % 4]) idx += inc;
    return idx > 3;
}

/* emp_piece.h:193-205 (operator==): orientations of b step by 2^sim(b) */
static int pieces_equal(const op_puzzle *p, uint32_t a, uint32_t b)
{
    if (a == b) return 1;
    uint32_t inc = 1u << p->sim[b];
    for (uint32_t o = 0; o <= 3; o += inc)
        if (compare_to(p, a, b, o)) return 1;
    return 0;
}

static void setf(char *err, size_t len, const char *msg)
{
    if (err && len) { strncpy(err, msg, len - 1); err[len - 1] = 0; }
}

op_puzzle *op_puzzle_create(uint32_t width, uint32_t height, const uint8_t *colours,
                            char *err, size_t err_len)
{
    if (width < 2 || height < 2 || width * height > OP_MAXN) {
        setf(err, err_len, "unsupported puzzle size");
        return NULL;
    }
    op_puzzle *p = (op_puzzle *)calloc(1, sizeof(op_puzzle));
    p->w = width; p->h = height; p->n = width * height;
    uint32_t expect[3] = {(width - 2) * (height - 2), 2 * (width - 2 + height - 2), 4};
    for (uint32_t i = 0; i < p->n; ++i) {
        uint32_t z = 0;
        for (int s = 0; s < 4; ++s) {
            p->col[i][s] = colours[4 * i + s];
            z += colours[4 * i + s] == 0;
            if (colours[4 * i + s] > p->max_color) p->max_color = colours[4 * i + s];
        }
        if (z > 2) { setf(err, err_len, "piece with more than 2 frame sides"); free(p); return NULL; }
        p->kind[i] = (uint8_t)z;                       /* emp_piece.h:122-131 */
        p->sim[i] = auto_similarity(p->col[i]);
        p->kind_index[i] = p->nb_kind[z]++;            /* emp_piece_db.h:540-610 */
        p->members[z][p->kind_index[i]] = i;
    }
    for (int k = 0; k < 3; ++k)
        if (p->nb_kind[k] != expect[k]) {
            setf(err, err_len, "piece kind counts do not match the puzzle size");
            free(p);
            return NULL;
        }
    p->border_id = p->max_color + 1;                   /* emp_piece_db.h:620-621 */
    p->cs = nb_bits(p->border_id);
    p->id_size = nb_bits(p->n - 1);
    p->dumped_id_size = nb_bits(p->n);
    p->max_code = 0;                                   /* emp_piece_db.h:739-748 */
    for (uint32_t l = 0; l < 4; ++l)
        p->max_code = (p->max_code << p->cs) | (l != 2 ? p->border_id : p->max_color);
    for (int k = 0; k < 3; ++k) {
        p->kind_bits[k] = 4 * p->nb_kind[k];
        p->kind_words[k] = (p->kind_bits[k] + 63) / 64;
        p->binary[k] = (uint32_t *)calloc(4 * p->nb_kind[k] + 1, sizeof(uint32_t));
    }
    /* binary pieces, emp_piece_db.h:751-764 and emp_piece.h:223-246 */
    for (uint32_t i = 0; i < p->n; ++i) {
        for (uint32_t o = 0; o < 4; ++o) {
            uint32_t r = (i << 2) | o;
            for (uint32_t l = 0; l < 4; ++l) {
                r <<= p->cs;
                uint32_t c = p->col[i][((3 - l) + o) % 4];
                r |= c ? c : p->border_id;
            }
            p->binary[p->kind[i]][p->kind_index[i] * 4 + o] = r;
        }
    }
    /* identical pieces, emp_piece_db.h:528-540 */
    for (uint32_t a = 0; a < p->n; ++a)
        for (uint32_t b = 0; b < p->n; ++b) {
            if (b == a) break;
            if (pieces_equal(p, a, b)) {
                p->twins[a][b >> 3] |= (uint8_t)(1u << (b & 7));
                p->twins[b][a >> 3] |= (uint8_t)(1u << (a & 7));
                p->has_identical = 1;
            }
        }
    /* identical masks, emp_piece_db.h:830-884 */
    for (int k = 0; k < 3; ++k) {
        uint32_t nw = p->kind_words[k];
        p->idmask[k] = (uint64_t *)calloc((size_t)p->kind_bits[k] * nw + 1, sizeof(uint64_t));
        for (uint32_t e = 0; e < p->kind_bits[k]; ++e) {
            uint64_t *m = p->idmask[k] + (size_t)e * nw;
            for (uint32_t b = 0; b < p->kind_bits[k]; ++b) bf_set1(m, b);
            bf_clr(m, e);
        }
    }
    for (uint32_t a = 0; a < p->n; ++a) {
        int k = p->kind[a];
        uint32_t nw = p->kind_words[k];
        for (uint32_t b = 0; b < p->n; ++b) {
            if (!(p->twins[a][b >> 3] & (1u << (b & 7)))) continue;
            for (uint32_t co = 0; co < 4; ++co) {
                if (!compare_to(p, a, b, co)) continue;
                for (uint32_t o = 0; o < 4; ++o) {
                    uint32_t e = p->kind_index[a] * 4 + o;
                    uint32_t e2 = p->kind_index[b] * 4 + (co + o) % 4;
                    if (e2 < p->kind_bits[k]) bf_clr(p->idmask[k] + (size_t)e * nw, e2);
                    else p->id_out_of_range = 1; /* the reference writes outside its bitfield here */
                }
            }
        }
    }
    return p;
}

static void build_table(op_puzzle *p)
{
    if (p->table_off) return;
    uint32_t nc = p->max_code + 1;
    p->table_off = (uint32_t *)malloc(sizeof(uint32_t) * nc);
    p->table_kind = (uint8_t *)calloc(nc, 1);
    for (uint32_t i = 0; i < nc; ++i) p->table_off[i] = UINT32_MAX;
    uint64_t total = 0;
    uint32_t B = p->border_id, cs = p->cs;
    /* emp_piece_db.h:770-819: only codes with at most two frame slots */
    for (uint32_t c1 = 0; c1 <= B; ++c1)
        for (uint32_t c2 = 0; c2 <= B; ++c2)
            for (uint32_t c3 = 0; c3 <= B; ++c3)
                for (uint32_t c4 = 0; c4 <= B; ++c4) {
                    uint32_t nb = (c1 == B) + (c2 == B) + (c3 == B) + (c4 == B);
                    if (nb > 2) continue;
                    uint32_t code = ((((c1 << cs) | c2) << cs | c3) << cs) | c4;
                    p->table_off[code] = (uint32_t)total;
                    p->table_kind[code] = (uint8_t)nb;
                    total += p->kind_words[nb];
                }
    p->table_words = total;
    p->table_pool = (uint64_t *)calloc(total + 1, sizeof(uint64_t));
    /* emp_piece_db.h:1267-1312 */
    for (uint32_t i = 0; i < p->n; ++i) {
        uint32_t inc = 1u << p->sim[i];
        for (uint32_t o = 0; o <= 3; o += inc) {
            uint32_t e = p->kind_index[i] * 4 + o;
            for (uint32_t sk = 0; sk <= 15; ++sk) {
                uint32_t code = 0, nb = 0;
                for (uint32_t s = 0; s < 4; ++s) {
                    if (!(sk & (1u << s))) continue;
                    uint32_t c = p->col[i][(s + o) % 4];
                    if (!c) { c = p->border_id; ++nb; }
                    code |= c << (p->cs * ((s + 2) % 4));
                }
                if (nb == p->kind[i]) bf_set1(p->table_pool + p->table_off[code], e);
            }
        }
    }
}

void op_puzzle_destroy(op_puzzle *p)
{
    if (!p) return;
    for (int k = 0; k < 3; ++k) { free(p->binary[k]); free(p->idmask[k]); }
    free(p->table_off); free(p->table_kind); free(p->table_pool);
    free(p);
}

int op_has_identical(const op_puzzle *p) { return p->has_identical; }
uint32_t op_nb_kind(const op_puzzle *p, uint32_t kind) { return kind < 3 ? p->nb_kind[kind] : 0; }
uint32_t op_kind_index(const op_puzzle *p, uint32_t i) { return i < p->n ? p->kind_index[i] : UINT32_MAX; }
uint32_t op_piece_of(const op_puzzle *p, uint32_t kind, uint32_t ki)
{
    return (kind < 3 && ki < p->nb_kind[kind]) ? p->members[kind][ki] : UINT32_MAX;
}
uint32_t op_border_color_id(const op_puzzle *p) { return p->border_id; }
uint32_t op_color_id_size(const op_puzzle *p) { return p->cs; }
uint32_t op_orientation_step(const op_puzzle *p, uint32_t i) { return 1u << p->sim[i]; }

uint32_t op_identical_mask(const op_puzzle *p, uint32_t kind, uint32_t t, uint64_t *out, uint32_t max_words)
{
    if (kind > 2 || t >= p->kind_bits[kind]) return 0;
    uint32_t nw = p->kind_words[kind];
    for (uint32_t i = 0; i < nw && i < max_words; ++i) out[i] = p->idmask[kind][(size_t)t * nw + i];
    return nw;
}

uint32_t op_table_entry(const op_puzzle *p, uint32_t code, uint64_t *out, uint32_t max_words)
{
    build_table((op_puzzle *)p);
    if (code > p->max_code || p->table_off[code] == UINT32_MAX) return 0;
    uint32_t k = p->table_kind[code];
    for (uint32_t i = 0; i < p->kind_words[k] && i < max_words; ++i) out[i] = p->table_pool[p->table_off[code] + i];
    return p->kind_bits[k];
}

/* ------------------------------------------------------------------ */
/* strategy orders                                                     */
void op_order_basic(uint32_t w, uint32_t h, uint32_t *order) /* emp_basic_strategy_generator.h:44-53 */
{
    uint32_t k = 0;
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) order[k++] = y * w + x;
}

void op_order_spiral(uint32_t w, uint32_t h, uint32_t *order) /* emp_spiral_strategy_generator.h:52-100 */
{
    uint8_t used[OP_MAXN];
    memset(used, 0, sizeof(used));
    uint32_t x = 0, y = 0, n = w * h;
    for (uint32_t i = 0; i < n; ++i) {
        used[y * w + x] = 1;
        order[i] = y * w + x;
        if (n > i + 1) {
            if (x >= y) {
                if (x + 1 < w && !used[y * w + x + 1]) x = x + 1;
                else if (y + 1 < h && !used[(y + 1) * w + x]) y = y + 1;
                else x = x - 1;
            } else {
                if (x && !used[y * w + x - 1]) x = x - 1;
                else if (y && !used[(y - 1) * w + x]) y = y - 1;
                else x = x + 1;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* emp_strategy restatement                                            */
typedef struct {
    const op_puzzle *p;
    uint32_t n;
    uint32_t kind[OP_MAXN + 1];
    uint32_t piece_info[OP_MAXN + 1];
    uint32_t nb_pos[OP_MAXN + 1][4];
    uint32_t nb_mask[OP_MAXN + 1][4];
    uint64_t *avail_trans;   /* [n][maxw] */
    uint64_t *avail_pieces;  /* [n][maxw] */
    const uint64_t *prev_avail[OP_MAXN + 1];
    uint64_t init_avail[3][16];
    uint32_t maxw;
    const uint32_t *order;
    uint32_t index_of[OP_MAXN];
} bt_state;

static void bt_init(bt_state *s, const op_puzzle *p, const uint32_t *order)
{
    memset(s, 0, sizeof(*s));
    s->p = p; s->n = p->n; s->order = order;
    s->maxw = 1;
    for (int k = 0; k < 3; ++k) if (p->kind_words[k] > s->maxw) s->maxw = p->kind_words[k];
    s->avail_trans = (uint64_t *)calloc((size_t)(s->n + 1) * s->maxw, sizeof(uint64_t));
    s->avail_pieces = (uint64_t *)calloc((size_t)(s->n + 1) * s->maxw, sizeof(uint64_t));
    for (int k = 0; k < 3; ++k)
        for (uint32_t b = 0; b < p->kind_bits[k]; ++b) bf_set1(s->init_avail[k], b);
    for (uint32_t i = 0; i < s->n; ++i) s->index_of[order[i]] = i;
    uint32_t cs = p->cs;
    uint32_t cmask = (1u << cs) - 1;
    uint32_t n = s->n, w = p->w, h = p->h;
    /* fake frame position, emp_strategy.h:194-204 */
    uint32_t fake = 0;
    for (uint32_t l = 0; l < 4; ++l) {
        fake = (fake << cs) | p->border_id;
        s->nb_pos[n][(l + 2) % 4] = n;
        s->nb_mask[n][(l + 2) % 4] = l != 2 ? cmask << (cs * l) : 0;
    }
    s->piece_info[n] = fake;
    const uint64_t *prev[3] = {s->init_avail[0], s->init_avail[1], s->init_avail[2]};
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t pos = order[i], x = pos % w, y = pos / w;
        int xb = x == 0 || x == w - 1, yb = y == 0 || y == h - 1;
        uint32_t k = (xb || yb) ? ((!xb || !yb) ? K_BORDER : K_CORNER) : K_CENTER;
        s->kind[i] = k;
        s->prev_avail[i] = prev[k];
        prev[k] = s->avail_pieces + (size_t)i * s->maxw;
        /* neighbour accessors, emp_strategy.h:232-262 */
        s->nb_pos[i][0] = y > 0 ? s->index_of[pos - w] : n;
        s->nb_mask[i][0] = cmask << (cs * 2);
        s->nb_pos[i][3] = x > 0 ? s->index_of[pos - 1] : n;
        s->nb_mask[i][3] = cmask << (cs * 1);
        s->nb_pos[i][2] = y < h - 1 ? s->index_of[pos + w] : n;
        s->nb_mask[i][2] = cmask << (cs * 0);
        s->nb_pos[i][1] = x < w - 1 ? s->index_of[pos + 1] : n;
        s->nb_mask[i][1] = cmask << (cs * 3);
    }
}

static void bt_free(bt_state *s) { free(s->avail_trans); free(s->avail_pieces); }

/* emp_strategy.h:291-296 with emp_position_strategy.h:172-186 */
static void bt_compute(bt_state *s, uint32_t i)
{
    uint64_t *at = s->avail_trans + (size_t)i * s->maxw;
    if (i == s->n) { memset(at, 0, sizeof(uint64_t) * s->maxw); return; }
    uint32_t code = 0;
    for (int d = 0; d < 4; ++d) code |= s->piece_info[s->nb_pos[i][d]] & s->nb_mask[i][d];
    const op_puzzle *p = s->p;
    uint32_t k = s->kind[i];
    if (code > p->max_code || p->table_off[code] == UINT32_MAX) {
        memset(at, 0, sizeof(uint64_t) * s->maxw);
        return;
    }
    const uint64_t *tab = p->table_pool + p->table_off[code];
    const uint64_t *prev = s->prev_avail[i];
    for (uint32_t j = 0; j < p->kind_words[k]; ++j) at[j] = tab[j] & prev[j];
}

/* emp_position_strategy.h:189-202 */
static void bt_select(bt_state *s, uint32_t i, uint32_t t)
{
    const op_puzzle *p = s->p;
    uint32_t k = s->kind[i], nw = p->kind_words[k];
    uint64_t *ap = s->avail_pieces + (size_t)i * s->maxw;
    uint64_t *at = s->avail_trans + (size_t)i * s->maxw;
    memcpy(ap, s->prev_avail[i], sizeof(uint64_t) * nw);
    for (uint32_t b = 0; b < 4; ++b) bf_clr(ap, (t & ~3u) + b);
    if (!p->has_identical) bf_clr(at, t);
    else {
        const uint64_t *m = p->idmask[k] + (size_t)t * nw;
        for (uint32_t j = 0; j < nw; ++j) at[j] &= m[j];
    }
}

static uint32_t bt_next(bt_state *s, uint32_t i)
{
    if (i == s->n) return 0;
    return bf_ffs(s->avail_trans + (size_t)i * s->maxw, s->p->kind_words[s->kind[i]]);
}

static size_t append(char *buf, size_t len, size_t pos, const char *txt)
{
    if (!buf || !len) return pos;
    size_t l = strlen(txt);
    if (pos + l + 1 > len) return pos;
    memcpy(buf + pos, txt, l + 1);
    return pos + l;
}

static void board_string(const bt_state *s, uint32_t upto, char *out)
{
    const op_puzzle *p = s->p;
    char tmp[16];
    int width = snprintf(tmp, sizeof(tmp), "%u", p->n) + 1;
    size_t L = (size_t)width * p->n;
    memset(out, '-', L);
    out[L] = 0;
    for (uint32_t i = 0; i <= upto && i < p->n; ++i) {
        uint32_t b = s->piece_info[i] >> (4 * p->cs);
        uint32_t pos = s->order[i];
        char cell[16];
        snprintf(cell, sizeof(cell), "%*u%c", width - 1, (b >> 2) + 1, "NESW"[b & 3]);
        memcpy(out + (size_t)pos * width, cell, (size_t)width);
    }
}

typedef struct { FILE *f; uint32_t nbits; uint64_t *words; uint32_t nwords; } dumper;

static void dump_open(dumper *d, const char *path, const op_puzzle *p, const uint32_t *order)
{
    memset(d, 0, sizeof(*d));
    if (!path) return;
    d->f = fopen(path, "wb");
    if (!d->f) return;
    uint32_t hdr[4] = {1, p->w, p->h, 1};
    fwrite(hdr, 4, 4, d->f);
    for (uint32_t i = 0; i < p->n; ++i) {
        uint32_t xy[2] = {order[i] % p->w, order[i] / p->w};
        fwrite(xy, 4, 2, d->f);
    }
    d->nbits = p->n * (p->id_size + 2);
    d->nwords = (d->nbits + 63) / 64;
    d->words = (uint64_t *)calloc(d->nwords, 8);
}

static void dump_solution(dumper *d, const bt_state *s, uint64_t nodes) /* emp_strategy.h:268-276 */
{
    if (!d->f) return;
    const op_puzzle *p = s->p;
    uint32_t fw = p->id_size + 2;
    memset(d->words, 0, 8 * (size_t)d->nwords);
    for (uint32_t i = 0; i < p->n; ++i) {
        uint32_t v = s->piece_info[i] >> (4 * p->cs);
        for (uint32_t b = 0; b < fw; ++b)
            if ((v >> b) & 1) bf_set1(d->words, i * fw + b);
    }
    fwrite(d->words, 8, d->nwords, d->f);
    fwrite(&nodes, 8, 1, d->f);
}

static void dump_close(dumper *d, uint64_t total)
{
    if (!d->f) return;
    fwrite(&total, 8, 1, d->f);
    fclose(d->f);
    free(d->words);
}

static int bt_run_impl(op_puzzle *p, const uint32_t *order, const uint16_t *situation, uint32_t placed,
                       uint64_t node_limit, op_bt_result *out, const char *results_bin, char *maxlog,
                       size_t maxlog_len);

int op_bt_run(op_puzzle *p, const uint32_t *order, uint64_t node_limit, op_bt_result *out,
              const char *results_bin, char *maxlog, size_t maxlog_len)
{
    return bt_run_impl(p, order, NULL, 0, node_limit, out, results_bin, maxlog, maxlog_len);
}

int op_bt_resume(op_puzzle *p, const uint32_t *order, const uint16_t *situation, uint32_t placed,
                 uint64_t node_limit, op_bt_result *out, const char *results_bin)
{
    if (!placed || placed >= p->n) return -1;
    return bt_run_impl(p, order, situation, placed, node_limit, out, results_bin, NULL, 0);
}

static int bt_run_impl(op_puzzle *p, const uint32_t *order, const uint16_t *situation, uint32_t placed,
                       uint64_t node_limit, op_bt_result *out, const char *results_bin, char *maxlog,
                       size_t maxlog_len)
{
    build_table(p);
    bt_state s;
    bt_init(&s, p, order);
    memset(out, 0, sizeof(*out));
    for (uint32_t i = 0; i < OP_MAXN; ++i) out->first_board[i] = 0xFFFFFFFFu;
    dumper d;
    dump_open(&d, results_bin, p, order);
    size_t lp = 0;
    if (maxlog && maxlog_len) maxlog[0] = 0;
    char *board = (char *)malloc(8 * OP_MAXN + 8);
    char line[64];
    uint32_t n = s.n, l_max = 0, idx = 0;
    uint64_t nodes = 0, sols = 0;
    int cont = 1;
    if (placed) {
        /* emp_strategy.h:418-467 (set_initial_state): each placed level takes its
         * candidates in order up to the situation's transition, applying select_piece
         * to every one tried; the search then starts at the LAST placed level (the
         * loop steps back from the first empty position), whose candidate set
         * specific_run recomputes from the start */
        for (uint32_t l = 0; l < placed; ++l) {
            bt_compute(&s, l);
            uint32_t t;
            do {
                uint32_t t1 = bt_next(&s, l);
                if (!t1) { free(board); bt_free(&s); dump_close(&d, 0); return -2; }
                t = t1 - 1;
                bt_select(&s, l, t);
            } while (t != situation[l]);
            s.piece_info[l] = p->binary[s.kind[l]][t];
        }
        idx = placed - 1;
    }
    bt_compute(&s, idx);
    /* emp_strategy.h:343-410 */
    while (cont) {
        if (node_limit && nodes >= node_limit) { out->status = 1; break; }
        uint32_t t1 = bt_next(&s, idx);
        if (t1) {
            uint32_t t = t1 - 1;
            s.piece_info[idx] = p->binary[s.kind[idx]][t];
            bt_select(&s, idx, t);
            ++nodes;
            if (idx > l_max) {
                snprintf(line, sizeof(line), "New max : %u\n", idx);
                lp = append(maxlog, maxlog_len, lp, line);
                board_string(&s, idx, board);
                lp = append(maxlog, maxlog_len, lp, board);
                lp = append(maxlog, maxlog_len, lp, "\n");
                l_max = idx;
            }
            if (idx == n - 1) {
                ++sols;
                dump_solution(&d, &s, nodes);
                if (sols == 1) {
                    out->first_solution_nodes = nodes;
                    for (uint32_t i = 0; i < n; ++i) {
                        uint32_t b = s.piece_info[i] >> (4 * p->cs);
                        out->first_board[order[i]] = b;
                        uint32_t pi = b >> 2;
                        out->first_solution[i] = (uint16_t)((p->kind_index[pi] << 2) | (b & 3));
                    }
                }
            }
            ++idx;
            bt_compute(&s, idx);
        } else {
            if (idx < n) s.piece_info[idx] = 0;
            cont = idx > 1;
            --idx;
            if (cont && idx > l_max) {
                snprintf(line, sizeof(line), "New max : %u\n", idx);
                lp = append(maxlog, maxlog_len, lp, line);
                board_string(&s, idx, board);
                lp = append(maxlog, maxlog_len, lp, board);
                lp = append(maxlog, maxlog_len, lp, "\n");
                l_max = idx;
            }
        }
    }
    dump_close(&d, nodes);
    out->nodes = nodes;
    out->solutions = sols;
    out->max_index = l_max;
    free(board);
    bt_free(&s);
    return 0;
}

/* state at level `depth` after replaying a prefix (levels 0..depth-1) */
static void bt_replay(bt_state *s, const uint16_t *prefix, uint32_t depth)
{
    const op_puzzle *p = s->p;
    for (uint32_t i = 0; i < depth; ++i) {
        uint32_t k = s->kind[i], t = prefix[i], nw = p->kind_words[k];
        s->piece_info[i] = p->binary[k][t];
        uint64_t *ap = s->avail_pieces + (size_t)i * s->maxw;
        memcpy(ap, s->prev_avail[i], sizeof(uint64_t) * nw);
        for (uint32_t b = 0; b < 4; ++b) bf_clr(ap, (t & ~3u) + b);
    }
}

static int bt_subtree_state(bt_state *s, const uint16_t *prefix, uint32_t depth, uint64_t node_limit,
                            uint64_t *nodes_out, uint64_t *sols_out, uint64_t *kind_nodes)
{
    const op_puzzle *p = s->p;
    uint32_t n = s->n;
    for (uint32_t i = 0; i <= n; ++i) if (i < n) s->piece_info[i] = 0;
    bt_replay(s, prefix, depth);
    uint64_t nodes = 0, sols = 0;
    int status = 0;
    if (depth >= n) { *nodes_out = 0; *sols_out = 0; return 0; }
    uint32_t idx = depth;
    bt_compute(s, idx);
    for (;;) {
        if (node_limit && nodes >= node_limit) { status = 1; break; }
        uint32_t t1 = bt_next(s, idx);
        if (t1) {
            uint32_t t = t1 - 1;
            s->piece_info[idx] = p->binary[s->kind[idx]][t];
            bt_select(s, idx, t);
            ++nodes;
            if (kind_nodes) ++kind_nodes[s->kind[idx]];
            if (idx == n - 1) ++sols;
            ++idx;
            bt_compute(s, idx);
        } else {
            if (idx < n) s->piece_info[idx] = 0;
            if (idx == depth) break;
            --idx;
        }
    }
    *nodes_out = nodes;
    *sols_out = sols;
    return status;
}

int op_bt_subtree(op_puzzle *p, const uint32_t *order, const uint16_t *prefix, uint32_t depth,
                  uint64_t node_limit, uint64_t *nodes, uint64_t *solutions)
{
    build_table(p);
    bt_state s;
    bt_init(&s, p, order);
    int r = bt_subtree_state(&s, prefix, depth, node_limit, nodes, solutions, NULL);
    bt_free(&s);
    return r;
}

uint64_t op_bt_expand(op_puzzle *p, const uint32_t *order, uint32_t depth, uint16_t *prefixes,
                      uint64_t max_prefixes, uint64_t *nodes_out, uint64_t *sols_out)
{
    build_table(p);
    bt_state s;
    bt_init(&s, p, order);
    uint32_t n = s.n;
    if (depth < 1) depth = 1;
    if (depth > n) depth = n;
    uint64_t count = 0, nodes = 0, sols = 0;
    uint16_t path[OP_MAXN];
    uint32_t idx = 0;
    int cont = 1;
    bt_compute(&s, 0);
    /* emp_strategy.h:343-410 with the walk cut at `depth` */
    while (cont) {
        uint32_t t1 = (idx < depth) ? bt_next(&s, idx) : 0;
        if (t1) {
            uint32_t t = t1 - 1;
            s.piece_info[idx] = p->binary[s.kind[idx]][t];
            bt_select(&s, idx, t);
            path[idx] = (uint16_t)t;
            ++nodes;
            if (idx == n - 1) ++sols;
            if (idx == depth - 1) {
                if (prefixes && count < max_prefixes) memcpy(prefixes + count * depth, path, 2 * (size_t)depth);
                ++count;
            }
            ++idx;
            if (idx < depth) bt_compute(&s, idx);
        } else {
            if (idx < n) s.piece_info[idx] = 0;
            cont = idx > 1;
            --idx;
        }
    }
    *nodes_out = nodes;
    *sols_out = sols;
    bt_free(&s);
    return count;
}


/* Knuth's random-probe estimate of the exhaustive tree size (placements):
 * E[prod of branching factors] summed over levels.  Used only to size
 * workloads; it does not take part in any parity check. */
double op_bt_estimate(op_puzzle *p, const uint32_t *order, uint32_t probes, uint64_t seed,
                      double *per_level)
{
    build_table(p);
    bt_state s;
    bt_init(&s, p, order);
    uint32_t n = s.n;
    double total = 0;
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    for (uint32_t pr = 0; pr < probes; ++pr) {
        double weight = 1;
        for (uint32_t i = 0; i < n; ++i) s.piece_info[i] = 0;
        uint32_t idx = 0;
        bt_compute(&s, 0);
        for (;;) {
            /* candidates actually tried at this level (identical masks applied in order) */
            uint32_t cand[1024], nc = 0;
            uint64_t *at = s.avail_trans + (size_t)idx * s.maxw;
            uint64_t save[16];
            memcpy(save, at, sizeof(uint64_t) * s.maxw);
            uint32_t t1;
            while ((t1 = bt_next(&s, idx)) != 0) {
                cand[nc++] = t1 - 1;
                bt_select(&s, idx, t1 - 1);
                if (idx == 0) break;   /* position 0 keeps its first transition */
            }
            memcpy(at, save, sizeof(uint64_t) * s.maxw);
            if (!nc) break;
            weight *= nc;
            total += weight;
            if (per_level) per_level[idx] += weight;
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            uint32_t t = cand[x % nc];
            s.piece_info[idx] = p->binary[s.kind[idx]][t];
            bt_select(&s, idx, t);
            ++idx;
            if (idx == n) break;
            bt_compute(&s, idx);
        }
    }
    bt_free(&s);
    if (per_level) for (uint32_t i = 0; i < n; ++i) per_level[i] /= probes;
    return total / probes;
}

typedef struct {
    op_puzzle *p;
    const uint32_t *order;
    const uint16_t *prefixes;
    uint32_t depth;
    uint64_t end;
    uint64_t *next;
    pthread_mutex_t *mu;
    uint64_t nodes, sols;
    uint64_t *per_nodes, *per_sols, begin;
    uint64_t kind_nodes[3];
} par_job;

static void *par_worker(void *arg)
{
    par_job *j = (par_job *)arg;
    bt_state s;
    bt_init(&s, j->p, j->order);
    for (;;) {
        uint64_t i = __atomic_fetch_add(j->next, 1, __ATOMIC_RELAXED);
        if (i >= j->end) break;
        uint64_t nn = 0, ss = 0;
        bt_subtree_state(&s, j->prefixes + i * j->depth, j->depth, 0, &nn, &ss, j->kind_nodes);
        j->nodes += nn;
        j->sols += ss;
        if (j->per_nodes) j->per_nodes[i - j->begin] = nn;
        if (j->per_sols) j->per_sols[i - j->begin] = ss;
    }
    bt_free(&s);
    return NULL;
}

int op_bt_subtrees_parallel(op_puzzle *p, const uint32_t *order, const uint16_t *prefixes,
                            uint32_t depth, uint64_t begin, uint64_t end, int nthreads,
                            uint64_t *nodes, uint64_t *solutions, uint64_t *per_nodes,
                            uint64_t *per_solutions, uint64_t *kind_nodes)
{
    build_table(p);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    uint64_t next = begin;
    par_job *jobs = (par_job *)calloc((size_t)nthreads, sizeof(par_job));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].p = p; jobs[t].order = order; jobs[t].prefixes = prefixes; jobs[t].depth = depth;
        jobs[t].end = end; jobs[t].next = &next; jobs[t].per_nodes = per_nodes;
        jobs[t].per_sols = per_solutions; jobs[t].begin = begin;
        pthread_create(&th[t], NULL, par_worker, &jobs[t]);
    }
    uint64_t nn = 0, ss = 0;
    for (int t = 0; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        nn += jobs[t].nodes;
        ss += jobs[t].sols;
        if (kind_nodes)
            for (int k = 0; k < 3; ++k) kind_nodes[k] += jobs[t].kind_nodes[k];
    }
    *nodes = nn;
    *solutions = ss;
    free(jobs);
    free(th);
    return 0;
}

/* ------------------------------------------------------------------ */
/* glutton max restatement                                             */
typedef struct {
    const op_puzzle *p;
    uint32_t size, n, level, max;
    uint32_t (*infos)[32];         /* triangular per-level infos */
    uint32_t position_index[OP_MAXN];
    uint32_t info_index[OP_MAXN];
    uint32_t played[OP_MAXN];
    uint32_t max_played[OP_MAXN];
    uint32_t avail[8];             /* 256 piece availability bits */
    uint16_t cnt[32][8];           /* per-lane piece infos */
    uint32_t (*cc)[4][32];         /* colour constraints [colour-1][side] */
    int offset[4];
    uint64_t placements, budget;
    int stop;
} gm_state;

static inline int gm_avail(const gm_state *g, uint32_t i) { return (g->avail[i >> 5] >> (i & 31)) & 1; }
static inline void gm_set_avail(gm_state *g, uint32_t i) { g->avail[i >> 5] |= 1u << (i & 31); }
static inline void gm_set_unavail(gm_state *g, uint32_t i) { g->avail[i >> 5] &= ~(1u << (i & 31)); }

/* CUDA_glutton_max_stack.h:339-343 */
static inline uint32_t *gm_info(gm_state *g, uint32_t level, uint32_t idx)
{
    uint32_t S = g->size;
    uint32_t base = (S * (S + 1) - (S - level) * (S - level + 1)) / 2;
    return g->infos[base + idx];
}

static inline int gm_any(const uint32_t *r) { for (int l = 0; l < 32; ++l) if (r[l]) return 1; return 0; }
static inline uint32_t gm_nb_info(const gm_state *g) { return g->size - g->level; }
static inline int gm_free(const gm_state *g, uint32_t pos) { return g->info_index[pos] < g->size - g->level; }

/* CUDA_glutton_max_stack.h:600-616 */
static void gm_clear_piece_info(gm_state *g)
{
    for (uint32_t l = 0; l < 32; ++l)
        for (uint32_t k = 0; k < 8; ++k) g->cnt[l][k] = gm_avail(g, 8 * l + k) ? 0 : 0xFFFF;
}

/* CUDA_glutton_max.h:260-287 */
static void gm_analyze(gm_state *g, const uint32_t *r)
{
    for (uint32_t l = 0; l < 32; ++l) {
        uint32_t v = r[l];
        for (uint32_t k = 0; k < 8; ++k) {
            g->cnt[l][k] = (uint16_t)(g->cnt[l][k] + (uint16_t)__builtin_popcount(v & 0xFu));
            v >>= 4;
        }
    }
}

typedef struct { uint32_t min, max, total; } gm_stats;

static void gm_update(uint32_t v, gm_stats *s) /* CUDA_glutton_max.h:221-229 */
{
    s->max = v > s->max ? v : s->max;
    s->min = v < s->min ? v : s->min;
    s->total += v;
}

/* One trial of candidate (info i, word w, bit b).  Returns 1 when valid.
 * With stats != NULL it also gathers the score of get_best_candidate
 * (CUDA_glutton_max.h:1010-1301); without it, it is the validity check of
 * remove_invalid_transitions (:745-954). */
static int gm_trial(gm_state *g, uint32_t i, uint32_t w, uint32_t b, gm_stats *st)
{
    const op_puzzle *p = g->p;
    uint32_t piece = 8 * w + b / 4, o = b % 4;
    uint32_t pos = g->position_index[i];
    uint32_t nb = gm_nb_info(g);
    ++g->placements;
    gm_set_unavail(g, piece);                    /* unvailability_lock_gard */
    gm_clear_piece_info(g);
    if (st) { st->min = 0xFFFFFFFFu; st->max = 0; st->total = 0; }
    uint32_t mask[32];
    for (uint32_t l = 0; l < 32; ++l) mask[l] = 0xFFFFFFFFu;
    mask[w] = ~(0xFu << (4 * (b / 4)));
    uint32_t related[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    uint32_t r[32];
    int valid = 1;
    /* apply_color_constraints, CUDA_glutton_max.h:531-612 */
    for (uint32_t s = 0; s < 4 && valid; ++s) {
        uint32_t c = p->col[piece][(s + o) % 4];
        if (!c) continue;
        uint32_t npos = (uint32_t)((int)pos + g->offset[s]);
        if (!gm_free(g, npos)) continue;
        uint32_t j = g->info_index[npos];
        uint32_t *cap = gm_info(g, g->level, j);
        for (uint32_t l = 0; l < 32; ++l) r[l] = cap[l] & (g->cc[c - 1][s][l] & mask[l]);
        if (!gm_any(r)) { valid = 0; break; }
        related[s] = j;
        gm_analyze(g, r);
        if (st) {
            uint32_t bits = 0;
            for (uint32_t l = 0; l < 32; ++l) bits += (uint32_t)__builtin_popcount(r[l]);
            gm_update(bits, st);
        }
    }
    /* apply_simple_mask over [0,i) then (i,nb), :471-526 and :869-908 */
    for (uint32_t j = 0; j < nb && valid; ++j) {
        if (j == i) continue;
        if (j == related[0] || j == related[1] || j == related[2] || j == related[3]) continue;
        uint32_t *cap = gm_info(g, g->level, j);
        for (uint32_t l = 0; l < 32; ++l) r[l] = cap[l] & mask[l];
        if (!gm_any(r)) { valid = 0; break; }
        gm_analyze(g, r);
        if (st) {
            uint32_t bits = 0;
            for (uint32_t l = 0; l < 32; ++l) bits += (uint32_t)__builtin_popcount(r[l]);
            gm_update(bits, st);
        }
    }
    if (valid) {
        /* piece coverage, :910-929 and :1196-1274 */
        gm_stats pst[32];
        for (uint32_t l = 0; l < 32; ++l) { pst[l].min = 0xFFFFFFFFu; pst[l].max = 0; pst[l].total = 0; }
        for (uint32_t k = 0; k < 8 && valid; ++k) {
            int all = 1;
            for (uint32_t l = 0; l < 32; ++l) if (!g->cnt[l][k]) { all = 0; break; }
            if (!all) { valid = 0; break; }
            if (st)
                for (uint32_t l = 0; l < 32; ++l)
                    if (gm_avail(g, 8 * l + k)) gm_update(g->cnt[l][k], &pst[l]);
        }
        if (valid && st) {
            uint32_t tot = 0, mn = 0xFFFFFFFFu, mx = 0;
            for (uint32_t l = 0; l < 32; ++l) {
                tot += pst[l].total;
                mn = pst[l].min < mn ? pst[l].min : mn;
                mx = pst[l].max > mx ? pst[l].max : mx;
            }
            st->total += tot;
            st->min = mn < st->min ? mn : st->min;
            st->max = mx > st->max ? mx : st->max;
        }
    }
    gm_set_avail(g, piece);
    return valid;
}

/* CUDA_glutton_max.h:624-714: lanes ascending, bits ascending over a
 * snapshot of the info words.  Calls fn for each candidate. */
typedef int (*gm_cand_fn)(gm_state *, uint32_t, uint32_t, uint32_t, void *);

static int gm_iterate(gm_state *g, uint32_t i, gm_cand_fn fn, void *ctx)
{
    uint32_t snap[32];
    memcpy(snap, gm_info(g, g->level, i), sizeof(snap));
    for (uint32_t l = 0; l < 32; ++l) {
        uint32_t v = snap[l];
        while (v) {
            uint32_t b = (uint32_t)__builtin_ctz(v);
            v &= ~(1u << b);
            if (fn(g, i, l, b, ctx)) return 1;
            if (g->stop) return 1;
        }
    }
    return 0;
}

typedef struct { int invalid_found; } rit_ctx;

static int rit_fn(gm_state *g, uint32_t i, uint32_t w, uint32_t b, void *vctx)
{
    rit_ctx *c = (rit_ctx *)vctx;
    if (g->budget && g->placements >= g->budget) { g->stop = 1; return 1; }
    if (!gm_trial(g, i, w, b, NULL)) {
        c->invalid_found = 1;
        gm_info(g, g->level, i)[w] &= ~(1u << b);   /* clear_invalid_bit */
    }
    return 0;
}

/* CUDA_glutton_max.h:745-954 */
static int gm_remove_invalid(gm_state *g)
{
    rit_ctx c;
    do {
        c.invalid_found = 0;
        for (uint32_t i = 0; i < gm_nb_info(g); ++i) {
            gm_iterate(g, i, rit_fn, &c);
            if (g->stop) return 1;
            if (!gm_any(gm_info(g, g->level, i))) return 0;
        }
    } while (c.invalid_found);
    return 1;
}

typedef struct { uint32_t best_info, best_total, best_minmax; } gbc_ctx;

static int gbc_fn(gm_state *g, uint32_t i, uint32_t w, uint32_t b, void *vctx)
{
    gbc_ctx *c = (gbc_ctx *)vctx;
    if (g->budget && g->placements >= g->budget) { g->stop = 1; return 1; }
    gm_stats st;
    if (!gm_trial(g, i, w, b, &st)) return 0;
    uint32_t minmax = (st.max << 16u) + st.min;
    if (st.total > c->best_total || (st.total == c->best_total && minmax > c->best_minmax) ||
        g->level == g->size - 1) {
        c->best_total = st.total;
        c->best_minmax = minmax;
        c->best_info = (w << 16u) | (b << 8u) | i;   /* generate_best_info */
    }
    return 0;
}

/* CUDA_glutton_max_stack.h:437-495 */
static void gm_push(gm_state *g, uint32_t info, uint32_t pos, uint32_t piece, uint32_t o)
{
    g->played[g->level] = (o << 16) | (piece << 8) | pos;
    gm_set_unavail(g, piece);
    ++g->level;
    if (g->level > g->max) {
        for (uint32_t l = 0; l <= g->max && l < g->size; ++l) g->max_played[l] = g->played[l];
        g->max = g->level;
    }
    uint32_t last = g->size - g->level;
    uint32_t last_pos = g->position_index[last];
    g->position_index[info] = info;
    /* swap_position_and_index */
    uint32_t tmp = g->info_index[pos]; g->info_index[pos] = g->info_index[last_pos]; g->info_index[last_pos] = tmp;
    tmp = g->position_index[info]; g->position_index[info] = g->position_index[last]; g->position_index[last] = tmp;
}

/* CUDA_glutton_max_stack.h:500-522 */
static uint32_t gm_pop(gm_state *g)
{
    uint32_t last = g->size - g->level;
    uint32_t info = g->position_index[last];
    uint32_t played = g->played[g->level - 1];
    uint32_t pos = played & 0xFFu;
    --g->level;
    gm_set_avail(g, (played >> 8) & 0xFFu);
    g->position_index[last] = pos;
    uint32_t pos2 = g->position_index[info];
    uint32_t tmp = g->info_index[pos]; g->info_index[pos] = g->info_index[pos2]; g->info_index[pos2] = tmp;
    tmp = g->position_index[info]; g->position_index[info] = g->position_index[last]; g->position_index[last] = tmp;
    return info;
}

/* CUDA_glutton_max.h:1306-1476 */
static void gm_apply(gm_state *g, uint32_t best)
{
    const op_puzzle *p = g->p;
    uint32_t i = best & 0xFFu, b = (best >> 8) & 0xFFu, w = best >> 16;
    gm_info(g, g->level, i)[w] &= ~(1u << b);
    uint32_t piece = 8 * w + b / 4, o = b % 4;
    uint32_t pos = g->position_index[i];
    uint32_t mask[32];
    for (uint32_t l = 0; l < 32; ++l) mask[l] = 0xFFFFFFFFu;
    mask[w] = ~(0xFu << (4 * (b / 4)));
    uint32_t nb = gm_nb_info(g);
    /* compute_next_level_position_info over [0,i) and [i+1, nb-1) */
    for (int pass = 0; pass < 2; ++pass) {
        uint32_t j0 = pass ? i + 1 : 0, j1 = pass ? nb - 1 : i;
        for (uint32_t j = j0; j < j1; ++j) {
            uint32_t *cap = gm_info(g, g->level, j), r[32];
            for (uint32_t l = 0; l < 32; ++l) r[l] = cap[l] & mask[l];
            if (!gm_any(r)) break;
            uint32_t *dst = gm_info(g, g->level + 1, j);
            memcpy(dst, r, sizeof(r));
        }
    }
    if (i < nb - 1 && g->level < g->size - 1) {
        uint32_t *cap = gm_info(g, g->level, nb - 1), r[32];
        for (uint32_t l = 0; l < 32; ++l) r[l] = cap[l] & mask[l];
        memcpy(gm_info(g, g->level + 1, i), r, sizeof(r));
        if (!gm_any(r)) return;
    }
    ++g->placements;
    gm_push(g, i, pos, piece, o);
    int invalid = 0;
    for (uint32_t s = 0; s < 4; ++s) {
        uint32_t c = p->col[piece][(s + o) % 4];
        if (!c) continue;
        uint32_t npos = (uint32_t)((int)pos + g->offset[s]);
        if (!gm_free(g, npos)) continue;
        uint32_t j = g->info_index[npos];
        uint32_t *cap = gm_info(g, g->level, j), r[32];
        for (uint32_t l = 0; l < 32; ++l) r[l] = cap[l] & g->cc[c - 1][s][l];
        if (!gm_any(r)) { invalid = 1; break; }
        uint32_t tgt = j < gm_nb_info(g) ? j : i;
        memcpy(gm_info(g, g->level, tgt), r, sizeof(r));
    }
    if (invalid) gm_pop(g);
}

/* The glutton search's first level: colour constraints and the initial capability of
 * every position (also the situation CUDA glutton wide prints). */
static gm_state *gm_setup(op_puzzle *p, uint64_t budget)
{
    gm_state *g = (gm_state *)calloc(1, sizeof(gm_state));
    g->p = p; g->size = p->n; g->n = p->n; g->budget = budget;
    uint32_t S = g->size;
    g->infos = (uint32_t(*)[32])calloc((size_t)S * (S + 1) / 2 + 1, sizeof(uint32_t[32]));
    g->cc = (uint32_t(*)[4][32])calloc(p->border_id + 1, sizeof(uint32_t[4][32]));
    g->offset[0] = -(int)p->w; g->offset[1] = 1; g->offset[2] = (int)p->w; g->offset[3] = -1;
    for (uint32_t i = 0; i < OP_MAXN; ++i) { g->played[i] = 0xFFFFFFFFu; g->max_played[i] = 0xFFFFFFFFu; }
    /* colour constraints, CUDA_common_glutton.h:111-146 */
    uint8_t present[256] = {0};
    for (uint32_t i = 0; i < p->n; ++i) for (int s = 0; s < 4; ++s) if (p->col[i][s]) present[p->col[i][s]] = 1;
    for (uint32_t c = 1; c <= p->max_color; ++c) {
        if (!present[c]) continue;
        for (uint32_t s = 0; s < 4; ++s) {
            uint32_t opp = (s + 2) % 4;
            for (uint32_t i = 0; i < p->n; ++i)
                for (uint32_t o = 0; o < 4; ++o)
                    if (p->col[i][(opp + o) % 4] == c) g->cc[c - 1][s][i / 8] |= 1u << (o + 4 * (i % 8));
        }
    }
    /* initial capability, CUDA_common_glutton.h:150-211; prepare_stack CUDA_glutton_max.h:120-156 */
    for (uint32_t i = 0; i < p->n; ++i) gm_set_avail(g, i);
    for (uint32_t pos = 0; pos < p->n; ++pos) {
        uint32_t x = pos % p->w, y = pos / p->w;
        uint32_t *cap = gm_info(g, 0, pos);
        int border = !x || !y || x == p->w - 1 || y == p->h - 1;
        int corner = (!x && !y) || (!x && y == p->h - 1) || (!y && x == p->w - 1) || (y == p->h - 1 && x == p->w - 1);
        if (corner) {
            uint32_t ci = (!x && !y) ? 0 : (!y ? 1 : (x ? 2 : 3));
            uint32_t b1 = ci, b2 = (ci + 3) % 4;       /* emp_FSM_info.h:281-301 */
            for (uint32_t k = 0; k < 4; ++k) {
                uint32_t piece = p->members[K_CORNER][k];
                for (uint32_t o = 0; o < 4; ++o)       /* emp_piece_corner.h:226-236 */
                    if (!p->col[piece][(b1 + o) % 4] && !p->col[piece][(b2 + o) % 4]) {
                        cap[piece / 8] |= 1u << (o + 4 * (piece % 8));
                        break;
                    }
            }
        } else if (border) {
            uint32_t bo = !y ? 0 : (x == p->w - 1 ? 1 : (y == p->h - 1 ? 2 : 3));
            for (uint32_t k = 0; k < p->nb_kind[K_BORDER]; ++k) {
                uint32_t piece = p->members[K_BORDER][k];
                uint32_t pb = 0;
                for (uint32_t s = 0; s < 4; ++s) if (!p->col[piece][s]) { pb = s; break; }
                uint32_t o = (pb + 4 - bo) % 4;          /* emp_piece_border.h:143-148 */
                cap[piece / 8] |= 1u << (o + 4 * (piece % 8));
            }
        } else {
            for (uint32_t k = 0; k < p->nb_kind[K_CENTER]; ++k) {
                uint32_t piece = p->members[K_CENTER][k];
                for (uint32_t o = 0; o < 4; ++o) cap[piece / 8] |= 1u << (o + 4 * (piece % 8));
            }
        }
        g->position_index[pos] = pos;
        g->info_index[pos] = pos;
    }
    return g;
}

/* CUDA glutton wide's situation (src/CUDA_glutton_wide.cu:27-37): level-0 infos of
 * the n positions, 32 words each, info index = position index. */
int op_gm_initial(op_puzzle *p, uint32_t *out)
{
    gm_state *g = gm_setup(p, 0);
    for (uint32_t pos = 0; pos < p->n; ++pos) memcpy(out + 32 * (size_t)pos, gm_info(g, 0, pos), 32 * sizeof(uint32_t));
    free(g->infos);
    free(g->cc);
    free(g);
    return 0;
}

int op_gm_run(op_puzzle *p, uint64_t budget, uint64_t push_budget, op_gm_result *out)
{
    memset(out, 0, sizeof(*out));
    gm_state *g = gm_setup(p, budget);
    /* kernel, CUDA_glutton_max.h:1522-1637 */
    int new_level = 1;
    uint32_t pop_index = 0;
    while (g->level < g->size) {
        if (g->stop) break;
        if (push_budget && out->pushes >= push_budget) { g->stop = 1; break; }
        if (!new_level && !gm_any(gm_info(g, g->level, pop_index))) {
            if (g->level == 0) { g->level = 0xFFFFFFFFu; break; }
            pop_index = gm_pop(g);
            ++out->pops;
            new_level = 0;
            continue;
        }
        ++out->levels_evaluated;
        int ok = gm_remove_invalid(g);
        if (g->stop) break;
        if (!ok) {
            if (g->level == 0) { g->level = 0xFFFFFFFFu; break; }
            pop_index = gm_pop(g);
            ++out->pops;
            new_level = 0;
            continue;
        }
        gbc_ctx c = {0xFFFFFFFFu, 0, 0};
        for (uint32_t i = 0; i < gm_nb_info(g) && !g->stop; ++i) gm_iterate(g, i, gbc_fn, &c);
        if (g->stop) break;
        if (c.best_info == 0xFFFFFFFFu) {
            if (g->level == 0) { g->level = 0xFFFFFFFFu; break; }
            pop_index = gm_pop(g);
            ++out->pops;
            new_level = 0;
            continue;
        }
        uint32_t lvl = g->level;
        gm_apply(g, c.best_info);
        if (g->level > lvl) ++out->pushes;
        new_level = 1;
    }
    out->placements = g->placements;
    out->max_level = g->max;
    out->level = g->level;
    out->status = g->level == g->size ? 0 : (g->stop ? 1 : 2);
    memcpy(out->played, g->played, sizeof(out->played));
    memcpy(out->max_played, g->max_played, sizeof(out->max_played));
    free(g->infos);
    free(g->cc);
    free(g);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Variable-space backtracker of the reference's CUDA_backtracker feature, as a
 * sequential restatement of its single-warp kernel (src/CUDA_backtracker.cu:67-178)
 * with the variables of emp_variable_generator::create_variables
 * (include/emp_variable_generator.h:335-525, no hints, empty situation) and the
 * transition vectors of system_equation_for_CUDA::prepare_transitions /
 * prepare_initial (include/system_equation_for_CUDA.h:70-173).
 *
 * A capability is 32 words: word 8*o + x/32, bit x%32 for (x, orientation o), where x
 * is a piece index for the first n capabilities (one per position, in row-major
 * order) and a position for the next n (one per piece).  Level l of the stack holds
 * 2n capabilities; levels above 0 start zeroed and keep whatever an earlier attempt
 * wrote, as the kernel's stack does (a piece already used at this level keeps a
 * stale capability, which the piece check reads). */
#define VS_W 32u

typedef struct { uint32_t pos, piece, o; } vs_var;

static void vs_clear(uint32_t *cap, uint32_t x, uint32_t o) { cap[8 * o + x / 32] &= ~(1u << (x % 32)); }
static void vs_set(uint32_t *cap, uint32_t x, uint32_t o) { cap[8 * o + x / 32] |= 1u << (x % 32); }

int op_vs_trace(op_puzzle *p, uint32_t max_events, uint32_t *ev_lane, uint32_t *ev_var, uint32_t *ev_step,
                uint32_t *n_events, uint32_t *solution_board, uint64_t max_selections)
{
    build_table(p);
    const uint32_t n = p->n, w = p->w, h = p->h, cs = p->cs, B = p->border_id;
    if (n > 256) return -1;
    /* variables per position, in the kind bitfield's ffs order */
    vs_var *vars = (vs_var *)calloc((size_t)n * 1024, sizeof(vs_var));
    uint32_t nv = 0;
    uint32_t *pos_first = (uint32_t *)calloc(n + 1, sizeof(uint32_t));
    for (uint32_t pos = 0; pos < n; ++pos) {
        const uint32_t x = pos % w, y = pos / w;
        pos_first[pos] = nv;
        const uint32_t E = x == w - 1 ? B : 0, N = y == 0 ? B : 0, W = x == 0 ? B : 0, S = y == h - 1 ? B : 0;
        const uint32_t code = (((((E << cs) | N) << cs) | W) << cs) | S;
        if (code > p->max_code || p->table_off[code] == UINT32_MAX) continue;
        const uint64_t *tab = p->table_pool + p->table_off[code];
        const uint32_t k = p->table_kind[code];
        for (uint32_t t = 0; t < p->kind_bits[k]; ++t) {
            if (!bf_get(tab, t)) continue;
            const uint32_t bin = p->binary[k][t] >> (4 * cs);
            vars[nv].pos = pos;
            vars[nv].piece = bin >> 2;
            vars[nv].o = bin & 3u;
            ++nv;
        }
    }
    pos_first[n] = nv;
    /* transition vectors, indexed by variable number */
    const size_t capw = (size_t)2 * n * VS_W;
    uint32_t *trans = (uint32_t *)malloc(sizeof(uint32_t) * capw * (nv ? nv : 1));
    memset(trans, 0xFF, sizeof(uint32_t) * capw * (nv ? nv : 1));
    int32_t *var_of = (int32_t *)malloc(sizeof(int32_t) * (size_t)n * 1024);
    for (size_t i = 0; i < (size_t)n * 1024; ++i) var_of[i] = -1;
    for (uint32_t v = 0; v < nv; ++v) var_of[vars[v].pos * 1024 + vars[v].o * 256 + vars[v].piece] = (int32_t)v;
    for (uint32_t v = 0; v < nv; ++v) {
        uint32_t *T = trans + capw * v;
        for (uint32_t u = pos_first[vars[v].pos]; u < pos_first[vars[v].pos + 1]; ++u) {
            vs_clear(T + VS_W * vars[v].pos, vars[u].piece, vars[u].o);
            vs_clear(T + VS_W * (n + vars[u].piece), vars[v].pos, vars[u].o);
        }
        for (uint32_t u = 0; u < nv; ++u) {
            if (vars[u].piece != vars[v].piece) continue;
            vs_clear(T + VS_W * (n + vars[v].piece), vars[u].pos, vars[u].o);
            vs_clear(T + VS_W * vars[u].pos, vars[v].piece, vars[u].o);
        }
    }
    /* incompatible neighbours (emp_variable_generator.h:558-621) */
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
            for (int dir = 0; dir < 2; ++dir) {
                if (dir == 0 && x + 1 >= w) continue;
                if (dir == 1 && y + 1 >= h) continue;
                const uint32_t p1 = y * w + x, p2 = dir == 0 ? p1 + 1 : p1 + w;
                const uint32_t side1 = dir == 0 ? 1u : 2u, side2 = dir == 0 ? 3u : 0u;
                for (uint32_t a = pos_first[p1]; a < pos_first[p1 + 1]; ++a)
                    for (uint32_t b = pos_first[p2]; b < pos_first[p2 + 1]; ++b) {
                        const vs_var *v1 = &vars[a], *v2 = &vars[b];
                        if (v1->piece == v2->piece) continue;
                        if (p->col[v1->piece][(side1 + v1->o) & 3] == p->col[v2->piece][(side2 + v2->o) & 3]) continue;
                        uint32_t *T1 = trans + capw * a, *T2 = trans + capw * b;
                        vs_clear(T1 + VS_W * p2, v2->piece, v2->o);
                        vs_clear(T1 + VS_W * (n + v2->piece), p2, v2->o);
                        vs_clear(T2 + VS_W * p1, v1->piece, v1->o);
                        vs_clear(T2 + VS_W * (n + v1->piece), p1, v1->o);
                    }
            }
    /* stack: n+1 levels of 2n capabilities, level 0 from prepare_initial */
    uint32_t *lev = (uint32_t *)calloc(capw * (n + 1), sizeof(uint32_t));
    for (uint32_t v = 0; v < nv; ++v) {
        vs_set(lev + VS_W * vars[v].pos, vars[v].piece, vars[v].o);
        vs_set(lev + VS_W * (n + vars[v].piece), vars[v].pos, vars[v].o);
    }
    uint32_t *stack_var = (uint32_t *)calloc(n, sizeof(uint32_t));
    uint32_t ne = 0, step = 0;
    uint64_t selections = 0;
    int found = 0;
    do {
        uint32_t *avail = lev + capw * step + VS_W * step;
        uint32_t lane = VS_W;
        for (uint32_t l = 0; l < VS_W; ++l)
            if (avail[l]) { lane = l; break; }
        if (lane == VS_W) { --step; continue; } /* step 0 wraps and ends the loop */
        const uint32_t bit = (uint32_t)__builtin_ctz(avail[lane]);
        const uint32_t var = (step << 10) | (lane << 5) | bit;
        const uint32_t piece = (lane % 8) * 32 + bit;
        if (ne < max_events) { ev_lane[ne] = lane; ev_var[ne] = var; ev_step[ne] = step; }
        ++ne;
        stack_var[step] = var;
        avail[lane] &= ~(1u << bit);
        if (step == n - 1) { found = 1; break; }
        if (max_selections && ++selections >= max_selections) break;
        const int32_t vi = var_of[var];
        const uint32_t *S = lev + capw * step, *T = trans + capw * (vi >= 0 ? vi : 0);
        uint32_t *R = lev + capw * (step + 1);
        int valid = vi >= 0;
        for (uint32_t q = step + 1; q < n && valid; ++q) {
            uint32_t any = 0, r[VS_W];
            for (uint32_t l = 0; l < VS_W; ++l) { r[l] = S[VS_W * q + l] & T[VS_W * q + l]; any |= r[l]; }
            if (any) memcpy(R + VS_W * q, r, sizeof(r));
            else valid = 0;
        }
        /* pieces below, then above, the selected one (src/CUDA_backtracker.cu:28-58,
         * called at :155-164 with the transition vector in the place of the situation
         * as well, so a piece's capability becomes the transition's own) */
        for (int pass = 0; pass < 2 && valid; ++pass) {
            const uint32_t q0 = pass ? piece + 1 : 0, q1 = pass ? n : piece;
            for (uint32_t q = q0; q < q1 && valid; ++q) {
                const uint32_t *Sq = T + VS_W * (n + q);
                uint32_t any_s = 0;
                for (uint32_t l = 0; l < VS_W; ++l) any_s |= Sq[l];
                if (!any_s) continue;
                uint32_t any = 0, r[VS_W];
                for (uint32_t l = 0; l < VS_W; ++l) { r[l] = Sq[l] & T[VS_W * (n + q) + l]; any |= r[l]; }
                if (any) memcpy(R + VS_W * (n + q), r, sizeof(r));
                else valid = 0;
            }
        }
        if (valid) {
            memset(R + VS_W * (n + piece), 0, sizeof(uint32_t) * VS_W);
            ++step;
        }
    } while (step < n);
    *n_events = ne;
    for (uint32_t i = 0; i < n; ++i) solution_board[i] = 0xFFFFFFFFu;
    if (found)
        for (uint32_t s = 0; s < n; ++s) {
            const uint32_t var = stack_var[s], lane = (var >> 5) & 31u, bit = var & 31u;
            solution_board[s] = (((lane % 8) * 32 + bit) << 2) | (lane / 8);
        }
    free(stack_var); free(lev); free(var_of); free(trans); free(pos_first); free(vars);
    return found ? 0 : 1;
}
