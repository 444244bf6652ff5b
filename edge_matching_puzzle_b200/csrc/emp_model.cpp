// Host-side puzzle model: see emp_model.h.
#include "emp_model.h"

#include <algorithm>
#include <cstring>

namespace emp {

namespace {

uint8_t auto_similarity(const std::array<uint8_t, 4>& c)  // emp_piece.h:144-157
{
    if (c[0] == c[2] && c[1] == c[3]) return c[0] == c[1] ? 2 : 1;
    return 0;
}

// emp_piece.h:208-220, "this" = a, argument = b rotated by o.  The sides of a
// are stepped by 2^similarity(a), which is why a half-symmetric piece compares
// only two of its sides.
bool compare_to(const PuzzleModel& m, uint32_t a, uint32_t b, uint32_t o)
{
    if (a == b) return true;
    uint32_t inc = 1u << m.similarity[a];
    uint32_t idx = 0;
    while (idx <= 3 && m.colours[a][idx] == m.colours[b][(idx + o) & 3]) idx += inc;
    return idx > 3;
}

// emp_piece.h:193-205: orientations of b step by 2^similarity(b).
bool pieces_equal(const PuzzleModel& m, uint32_t a, uint32_t b)
{
    if (a == b) return true;
    uint32_t inc = 1u << m.similarity[b];
    for (uint32_t o = 0; o <= 3; o += inc)
        if (compare_to(m, a, b, o)) return true;
    return false;
}

inline void set_bit(uint32_t* w, uint32_t i) { w[i >> 5] |= 1u << (i & 31); }
inline void clr_bit(uint32_t* w, uint32_t i) { w[i >> 5] &= ~(1u << (i & 31)); }

}  // namespace

bool build_model(uint32_t width, uint32_t height, const uint8_t* colours, PuzzleModel& m,
                 std::string& error)
{
    m = PuzzleModel();
    if (width < 2 || height < 2 || width * height > kMaxPieces) {
        error = "unsupported puzzle size (need 2 <= w,h and w*h <= 256)";
        return false;
    }
    m.width = width;
    m.height = height;
    m.n = width * height;
    m.colours.resize(m.n);
    m.kind.resize(m.n);
    m.similarity.resize(m.n);
    m.kind_index.resize(m.n);
    for (uint32_t i = 0; i < m.n; ++i) {
        uint32_t zeros = 0;
        for (uint32_t s = 0; s < 4; ++s) {
            m.colours[i][s] = colours[4 * i + s];
            zeros += colours[4 * i + s] == 0;
            m.max_colour = std::max<uint32_t>(m.max_colour, colours[4 * i + s]);
        }
        if (zeros > 2) {
            error = "piece " + std::to_string(i + 1) + " has more than two frame sides";
            return false;
        }
        m.kind[i] = static_cast<uint8_t>(zeros);
        m.similarity[i] = auto_similarity(m.colours[i]);
        m.kind_index[i] = static_cast<uint32_t>(m.members[zeros].size());
        m.members[zeros].push_back(i);
    }
    const uint32_t expect[3] = {(width - 2) * (height - 2), 2 * (width - 2 + height - 2), 4};
    for (uint32_t k = 0; k < 3; ++k)
        if (m.nb_kind(k) != expect[k]) {
            error = "piece kind counts do not match a " + std::to_string(width) + "x" +
                    std::to_string(height) + " puzzle";
            return false;
        }
    m.border_id = m.max_colour + 1;
    if (m.border_id > kMaxColourId) {
        error = "colour ids above 30 are not supported";
        return false;
    }
    // Every colour must appear an even number of times (emp_piece_db.h:898-910).
    std::vector<uint32_t> count(m.border_id + 1, 0);
    for (uint32_t i = 0; i < m.n; ++i)
        for (uint32_t s = 0; s < 4; ++s) count[m.colours[i][s]]++;
    for (uint32_t c = 1; c <= m.max_colour; ++c)
        if (count[c] % 2) {
            error = "Number of pieces edge with color should be multiple of 2 or the puzzle cannot be solved";
            return false;
        }
    for (uint32_t k = 0; k < 3; ++k) m.kind_words[k] = (4 * m.nb_kind(k) + 31) / 32;

    // identical pieces (emp_piece_db.h:528-540): a is compared to every piece
    // placed before it in the file
    std::vector<std::vector<uint8_t>> twin(m.n, std::vector<uint8_t>(m.n, 0));
    for (uint32_t a = 0; a < m.n; ++a)
        for (uint32_t b = 0; b < a; ++b)
            if (pieces_equal(m, a, b)) {
                twin[a][b] = twin[b][a] = 1;
                m.has_identical = true;
            }
    // identical masks (emp_piece_db.h:830-884)
    for (uint32_t k = 0; k < 3; ++k) {
        uint32_t bits = 4 * m.nb_kind(k), nw = m.kind_words[k];
        m.idmask[k].assign(static_cast<size_t>(bits) * nw, 0);
        for (uint32_t e = 0; e < bits; ++e) {
            uint32_t* w = &m.idmask[k][static_cast<size_t>(e) * nw];
            for (uint32_t b = 0; b < bits; ++b) set_bit(w, b);
            clr_bit(w, e);
        }
    }
    for (uint32_t a = 0; a < m.n; ++a) {
        uint32_t k = m.kind[a], bits = 4 * m.nb_kind(k), nw = m.kind_words[k];
        for (uint32_t b = 0; b < m.n; ++b) {
            if (!twin[a][b]) continue;
            for (uint32_t co = 0; co < 4; ++co) {
                if (!compare_to(m, a, b, co)) continue;
                for (uint32_t o = 0; o < 4; ++o) {
                    uint32_t e = m.kind_index[a] * 4 + o;
                    uint32_t e2 = m.kind_index[b] * 4 + ((co + o) & 3);
                    // e2 indexes b's own kind; when b is of another kind and its
                    // index lies past a's bitfield the reference writes outside
                    // the bitfield.  That write is dropped here (and in the oracle).
                    if (e2 < bits) clr_bit(&m.idmask[k][static_cast<size_t>(e) * nw], e2);
                    else m.identical_out_of_range = true;
                }
            }
        }
    }
    return true;
}

std::vector<uint32_t> order_basic(uint32_t w, uint32_t h)
{
    std::vector<uint32_t> o;
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) o.push_back(y * w + x);
    return o;
}

std::vector<uint32_t> order_spiral(uint32_t w, uint32_t h)  // emp_spiral_strategy_generator.h:52-100
{
    std::vector<uint8_t> used(w * h, 0);
    std::vector<uint32_t> o;
    uint32_t x = 0, y = 0, n = w * h;
    for (uint32_t i = 0; i < n; ++i) {
        used[y * w + x] = 1;
        o.push_back(y * w + x);
        if (n > i + 1) {
            if (x >= y) {
                if (x + 1 < w && !used[y * w + x + 1]) ++x;
                else if (y + 1 < h && !used[(y + 1) * w + x]) ++y;
                else --x;
            } else {
                if (x && !used[y * w + x - 1]) --x;
                else if (y && !used[(y - 1) * w + x]) --y;
                else ++x;
            }
        }
    }
    return o;
}

bool build_plan(const PuzzleModel& m, const std::vector<uint32_t>& order,
                std::vector<LevelPlan>& plan, std::string& error)
{
    if (order.size() != m.n) {
        error = "position order must list every position once";
        return false;
    }
    std::vector<int> level_of(m.n, -1);
    for (uint32_t i = 0; i < m.n; ++i) {
        if (order[i] >= m.n || level_of[order[i]] >= 0) {
            error = "position order must list every position once";
            return false;
        }
        level_of[order[i]] = static_cast<int>(i);
    }
    plan.assign(m.n, LevelPlan());
    for (uint32_t L = 0; L < m.n; ++L) {
        LevelPlan& lp = plan[L];
        uint32_t pos = order[L], x = pos % m.width, y = pos / m.width;
        bool xb = x == 0 || x == m.width - 1, yb = y == 0 || y == m.height - 1;
        lp.position = pos;
        lp.kind = (xb || yb) ? ((!xb || !yb) ? kBorder : kCorner) : kCenter;
        // frame sides of this position and neighbours placed earlier
        bool frame[4] = {y == 0, x == m.width - 1, y == m.height - 1, x == 0};
        int nbpos[4] = {y > 0 ? static_cast<int>(pos - m.width) : -1,
                        x + 1 < m.width ? static_cast<int>(pos + 1) : -1,
                        y + 1 < m.height ? static_cast<int>(pos + m.width) : -1,
                        x > 0 ? static_cast<int>(pos - 1) : -1};
        for (uint32_t s = 0; s < 4; ++s)
            if (nbpos[s] >= 0 && level_of[nbpos[s]] < static_cast<int>(L)) {
                lp.side[lp.nplaced] = static_cast<uint8_t>(s);
                lp.nb_level[lp.nplaced] = static_cast<uint8_t>(level_of[nbpos[s]]);
                ++lp.nplaced;
            }
        // base = allowed orientations whose frame sides are exactly the
        // position's frame sides (emp_piece_db.h:1281-1309 with nb_border == kind)
        uint32_t k = lp.kind;
        lp.base.assign(m.kind_words[k], 0);
        for (uint32_t ki = 0; ki < m.nb_kind(k); ++ki) {
            uint32_t p = m.members[k][ki];
            for (uint32_t o = 0; o < 4; ++o) {
                if (!m.allowed(p, o)) continue;
                bool ok = true;
                for (uint32_t s = 0; s < 4 && ok; ++s)
                    if (frame[s]) ok = m.colour(p, s, o) == 0;
                if (ok) set_bit(lp.base.data(), 4 * ki + o);
            }
        }
    }
    return true;
}

namespace {

inline void set_bit64(uint64_t* w, uint32_t i) { w[i >> 6] |= uint64_t(1) << (i & 63); }

void push64(std::vector<uint32_t>& b, uint64_t v)
{
    b.push_back(static_cast<uint32_t>(v));
    b.push_back(static_cast<uint32_t>(v >> 32));
}

void align(std::vector<uint32_t>& b, size_t words)
{
    while (b.size() % words) b.push_back(0);
}

}  // namespace

void build_device_tables(const PuzzleModel& m, const std::vector<LevelPlan>& plan, DeviceTables& t)
{
    t = DeviceTables();
    t.n = m.n;
    t.ncol = m.border_id + 1;
    for (uint32_t k = 0; k < 3; ++k) {
        t.kw[k] = (4 * m.nb_kind(k) + 63) / 64;
        t.aoff[k] = t.avail_words;
        t.avail_words += t.kw[k];
        t.max_kw = std::max(t.max_kw, t.kw[k]);
    }
    std::vector<uint32_t>& b = t.blob;
    b.assign(kHeaderWords, 0);
    // side masks per kind: bit (ki,o) when side s of piece ki@o shows colour c
    // (c = border_id for a frame side), for allowed orientations only
    std::array<std::vector<uint64_t>, 3> side;
    for (uint32_t k = 0; k < 3; ++k) {
        side[k].assign(static_cast<size_t>(4) * t.ncol * t.kw[k], 0);
        for (uint32_t ki = 0; ki < m.nb_kind(k); ++ki) {
            const uint32_t p = m.members[k][ki];
            for (uint32_t o = 0; o < 4; ++o) {
                if (!m.allowed(p, o)) continue;
                for (uint32_t s = 0; s < 4; ++s) {
                    uint32_t c = m.colour(p, s, o);
                    if (!c) c = m.border_id;
                    set_bit64(&side[k][(static_cast<size_t>(s) * t.ncol + c) * t.kw[k]], 4 * ki + o);
                }
            }
        }
    }
    // pair tables, one per distinct (kind, base, paired sides) class
    align(b, 4);
    t.pair_off = static_cast<uint32_t>(b.size());
    struct Key {
        uint32_t kind, arity, sa, sb;
        std::vector<uint32_t> base;
        bool operator==(const Key& o) const
        {
            return kind == o.kind && arity == o.arity && sa == o.sa && sb == o.sb && base == o.base;
        }
    };
    std::vector<std::pair<Key, uint32_t>> classes;
    std::vector<uint32_t> level_pair(m.n);
    for (uint32_t L = 0; L < m.n; ++L) {
        const LevelPlan& lp = plan[L];
        Key key{lp.kind, std::min<uint32_t>(lp.nplaced, 2), lp.nplaced > 0 ? lp.side[0] : 0u,
                lp.nplaced > 1 ? lp.side[1] : 0u, lp.base};
        uint32_t off = 0;
        bool found = false;
        for (const auto& c : classes)
            if (c.first == key) {
                off = c.second;
                found = true;
                break;
            }
        if (!found) {
            align(b, 4);
            off = static_cast<uint32_t>(b.size());
            const uint32_t k = key.kind, kw = t.kw[k];
            std::vector<uint64_t> base64(kw, 0);
            for (uint32_t i = 0; i < 4 * m.nb_kind(k); ++i)
                if ((lp.base[i >> 5] >> (i & 31)) & 1u) set_bit64(base64.data(), i);
            const uint32_t na = key.arity >= 1 ? t.ncol : 1, nb = key.arity >= 2 ? t.ncol : 1;
            for (uint32_t ca = 0; ca < na; ++ca)
                for (uint32_t cb = 0; cb < nb; ++cb)
                    for (uint32_t w = 0; w < kw; ++w) {
                        uint64_t v = base64[w];
                        if (key.arity >= 1) v &= side[k][(static_cast<size_t>(key.sa) * t.ncol + ca) * kw + w];
                        if (key.arity >= 2) v &= side[k][(static_cast<size_t>(key.sb) * t.ncol + cb) * kw + w];
                        push64(b, v);
                    }
            classes.push_back({key, off});
        }
        level_pair[L] = off;
    }
    // level descriptors
    align(b, 4);
    t.desc_off = static_cast<uint32_t>(b.size());
    b.resize(b.size() + kDescWords * static_cast<size_t>(m.n), 0);
    // transition info
    for (uint32_t k = 0; k < 3; ++k) {
        align(b, 2);
        t.tinfo_off[k] = static_cast<uint32_t>(b.size());
        const uint32_t bits = 4 * m.nb_kind(k);
        for (uint32_t e = 0; e < bits; ++e) {
            const uint32_t p = m.members[k][e >> 2], o = e & 3;
            uint32_t v = 0;
            for (uint32_t s = 0; s < 4; ++s) v |= m.colour(p, s, o) << (5 * s);
            // extra clears: bits the identical mask removes besides e itself,
            // restricted to allowed candidates (others never appear in a set)
            const uint32_t* im = &m.idmask[k][static_cast<size_t>(e) * m.kind_words[k]];
            for (uint32_t e2 = 0; e2 < bits; ++e2) {
                if (e2 == e || !m.allowed(m.members[k][e2 >> 2], e2 & 3)) continue;
                if (!((im[e2 >> 5] >> (e2 & 31)) & 1u)) {
                    v |= 1u << 20;
                    break;
                }
            }
            b.push_back(v);
        }
    }
    // side masks: only read for the third and fourth placed neighbour of a level
    for (uint32_t k = 0; k < 3; ++k) {
        align(b, 4);
        t.side_off[k] = static_cast<uint32_t>(b.size());
        for (uint64_t v : side[k]) push64(b, v);
    }
    for (uint32_t k = 0; k < 3; ++k) {
        align(b, 2);
        t.extra_off[k] = static_cast<uint32_t>(b.size());
        const uint32_t bits = 4 * m.nb_kind(k);
        for (uint32_t e = 0; e < bits; ++e) {
            const uint32_t* im = &m.idmask[k][static_cast<size_t>(e) * m.kind_words[k]];
            for (uint32_t w = 0; w < t.kw[k]; ++w) {
                uint64_t v = 0;
                for (uint32_t i = 0; i < 64; ++i) {
                    const uint32_t bit = 64 * w + i;
                    // bits past the kind's candidates stay 1, like the reference's all-ones init
                    const bool one = bit >= bits || ((im[bit >> 5] >> (bit & 31)) & 1u);
                    if (one) v |= uint64_t(1) << i;
                }
                push64(b, v);
            }
        }
    }
    align(b, 2);
    t.init_off = static_cast<uint32_t>(b.size());
    for (uint32_t k = 0; k < 3; ++k) {
        const uint32_t bits = 4 * m.nb_kind(k);
        for (uint32_t w = 0; w < t.kw[k]; ++w) {
            uint64_t v = 0;
            for (uint32_t i = 0; i < 64; ++i)
                if (w * 64 + i < bits) v |= uint64_t(1) << i;
            push64(b, v);
        }
    }
    align(b, 4);
    for (uint32_t L = 0; L < m.n; ++L) {
        const LevelPlan& lp = plan[L];
        uint32_t* d = &b[t.desc_off + kDescWords * L];
        const uint32_t k = lp.kind;
        const uint32_t arity = std::min<uint32_t>(lp.nplaced, 2);
        const uint32_t nextra = lp.nplaced - arity;
        // facing colour of the neighbour at side s sits at bits 5*((s+2)&3) of its stack word
        const uint32_t shift_a = arity > 0 ? 5 * ((lp.side[0] + 2u) & 3u) : 0u;
        const uint32_t shift_b = arity > 1 ? 5 * ((lp.side[1] + 2u) & 3u) : 0u;
        const uint32_t stride_b = arity > 1 ? 2 * t.kw[k] : 0u;
        const uint32_t stride_a = arity > 1 ? 2 * t.kw[k] * t.ncol : (arity > 0 ? 2 * t.kw[k] : 0u);
        d[0] = t.kw[k] | (k << 8) | (nextra << 13) | (t.aoff[k] << 16);
        d[1] = (arity > 0 ? lp.nb_level[0] : 0u) | ((arity > 1 ? lp.nb_level[1] : 0u) << 8) | (shift_a << 16) |
               (shift_b << 24);
        d[2] = level_pair[L];
        d[3] = stride_a | (stride_b << 16);
        d[4] = t.side_off[k];
        d[5] = t.tinfo_off[k];
        d[6] = t.extra_off[k];
        d[7] = (nextra > 0 ? lp.side[2] : 0u) | ((nextra > 1 ? lp.side[3] : 0u) << 2) |
               ((nextra > 0 ? lp.nb_level[2] : 0u) << 8) | ((nextra > 1 ? lp.nb_level[3] : 0u) << 16);
        for (uint32_t j = 0; j < 4; ++j) {
            const uint32_t lev = j < lp.nplaced ? lp.nb_level[j] : 0u;
            d[8 + j] = t.tinfo_off[plan[lev].kind];
        }
    }
    b[0] = 0x454D5034u;  // "EMP4": 64-bit candidate words, 16-word descriptors
    b[1] = t.n;
    b[2] = t.ncol;
    for (uint32_t k = 0; k < 3; ++k) {
        b[3 + k] = t.kw[k];
        b[6 + k] = t.aoff[k];
        b[10 + k] = t.side_off[k];
        b[15 + k] = t.tinfo_off[k];
        b[18 + k] = t.extra_off[k];
    }
    b[9] = t.avail_words;
    b[13] = t.pair_off;
    b[14] = t.desc_off;
    b[21] = t.init_off;
    b[22] = m.width;
    b[23] = m.height;
    b[24] = static_cast<uint32_t>(b.size());
    b[25] = t.max_kw;
    b[26] = t.side_off[0];  // words [0, side[0]) are what a kernel may stage in shared memory
}

namespace {
struct SplitMix64 {
    uint64_t s;
    uint64_t next()
    {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint32_t below(uint32_t bound) { return static_cast<uint32_t>(next() % bound); }
};
}  // namespace

void generate_puzzle(uint32_t w, uint32_t h, uint32_t B, uint32_t I, uint64_t seed, uint8_t* out)
{
    SplitMix64 r{seed};
    std::vector<uint32_t> hor(static_cast<size_t>(h) * (w - 1)), ver(static_cast<size_t>(h - 1) * w);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x + 1 < w; ++x)
            hor[y * (w - 1) + x] = (y == 0 || y == h - 1) ? 1 + r.below(B) : B + 1 + r.below(I);
    for (uint32_t y = 0; y + 1 < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
            ver[y * w + x] = (x == 0 || x == w - 1) ? 1 + r.below(B) : B + 1 + r.below(I);
    uint32_t n = w * h;
    std::vector<std::array<uint32_t, 4>> p(n);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            auto& c = p[y * w + x];
            c[0] = y == 0 ? 0 : ver[(y - 1) * w + x];
            c[1] = x == w - 1 ? 0 : hor[y * (w - 1) + x];
            c[2] = y == h - 1 ? 0 : ver[y * w + x];
            c[3] = x == 0 ? 0 : hor[y * (w - 1) + x - 1];
        }
    for (uint32_t i = n - 1; i > 0; --i) std::swap(p[i], p[r.below(i + 1)]);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t k = r.below(4);
        for (uint32_t s = 0; s < 4; ++s) out[4 * i + s] = static_cast<uint8_t>(p[i][(s + k) & 3]);
    }
}

}  // namespace emp
