// host_graph.cpp -- text ingest and query planning (host side of libgfsm).
//
// parse_text restates the reference parser's semantics (HnHelper.cuh:191-266
// parseValues, :283-381 fileParse) but runs multi-threaded over line-aligned
// chunks: the reference reads the file byte by byte on one thread.
// plan_query restates the reference's matching order and requirement table
// (HnGPU.cu:749-816 preProcessQuery, ccsr.cpp:98-219).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <thread>

#include "gfsm_internal.h"

namespace gfsm {

namespace {

enum LineKind : uint8_t { L_V, L_E, L_END, L_BAD };

// Tokenises one line the way parseValues does (HnHelper.cuh:233-263): digit
// runs accumulate into the current value slot with uint32 wrap-around, every
// other byte moves to the next slot, '\n' ends the line.
// Every non-digit byte moves to the next slot, so a slot receives at most
// one digit run: it is accumulated in a register and stored when the run's
// slot ends.
inline const char *scan_values(const char *s, const char *end, uint32_t *v, int nv) {
    uint32_t cur = 0, acc = 0;
    for (; s < end; ++s) {
        const uint32_t d = (uint32_t)(uint8_t)*s - (uint32_t)'0';
        if (d < 10u) {
            acc = acc * 10u + d;
            continue;
        }
        if ((int)cur < nv) v[cur] = acc;
        acc = 0;
        ++cur;
        if (*s == '\n') return s + 1;
    }
    if ((int)cur < nv) v[cur] = acc;
    return s;
}

struct ChunkOut {
    std::vector<uint32_t> es, ed, el;      // edge lines
    std::vector<uint32_t> vid, vlab;       // vertex lines
    uint64_t first_stop = UINT64_MAX;      // byte offset of the first 't' or bad line
    LineKind stop_kind = L_END;
    uint64_t first_e = UINT64_MAX;         // byte offset of the first 'e' line
    uint64_t last_v = 0;                   // byte offset of the last 'v' line (+1), 0 if none
    // per-line order for validation: offsets of the first 'v' after an 'e'
    uint64_t first_v_after_e = UINT64_MAX;
};

void scan_chunk(const char *buf, uint64_t b, uint64_t e, uint64_t len, ChunkOut &o) {
    const char *end = buf + len, *s = buf + b, *const stop = buf + e;
    {
        // room for the chunk's lines at the mean length of its first 64 KiB
        const char *probe = s + std::min<uint64_t>(e - b, 1u << 16);
        uint64_t lines = 1;
        for (const char *x = s; x < probe; ++x) lines += *x == '\n';
        const uint64_t guess = (e - b) / std::max<uint64_t>(1, (uint64_t)(probe - s) / lines) + 16;
        o.es.reserve(guess);
        o.ed.reserve(guess);
        o.el.reserve(guess);
    }
    while (s < stop) {
        const uint64_t pos = (uint64_t)(s - buf);
        const char ch = *s;
        if (ch == 't') {
            bool ok = (uint64_t)(end - s) >= 6 && !strncmp(s, "t # -1", 6);
            o.first_stop = pos;
            o.stop_kind = ok ? L_END : L_BAD;
            return;
        }
        if (ch != 'v' && ch != 'e') {
            o.first_stop = pos;
            o.stop_kind = L_BAD;
            return;
        }
        // the values start two bytes in ("e " / "v "); a line that ends
        // sooner has none
        uint32_t v[3] = {0, 0, 0};
        if (s + 1 >= end) s = end;
        else if (s[1] == '\n') s += 2;
        else s = scan_values(s + 2, end, v, 3);
        if (ch == 'v') {
            o.vid.push_back(v[0]);
            o.vlab.push_back(v[1]);
            o.last_v = pos + 1;
            if (o.first_e != UINT64_MAX && o.first_v_after_e == UINT64_MAX) o.first_v_after_e = pos;
        } else {
            if (o.first_e == UINT64_MAX) o.first_e = pos;
            o.es.push_back(v[0]);
            o.ed.push_back(v[1]);
            o.el.push_back(v[2]);
        }
    }
}

}  // namespace

gfsm_status FileBytes::open(const char *path) {
    close();
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return GFSM_ERR_MISSING_FILE;  // HnHelper.cuh:289-294
    struct stat sb {};
    if (fstat(fd, &sb) == 0 && S_ISREG(sb.st_mode) && sb.st_size > 0) {
        void *m = mmap(nullptr, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m != MAP_FAILED) {
            map_ = m;
            len_ = (uint64_t)sb.st_size;
            ::close(fd);
            return GFSM_OK;
        }
    }
    // not mappable (a pipe, a special file): read it whole
    char tmp[1 << 16];
    for (;;) {
        const ssize_t got = ::read(fd, tmp, sizeof(tmp));
        if (got < 0 && errno == EINTR) continue;
        if (got <= 0) break;
        buf_.append(tmp, (size_t)got);
    }
    ::close(fd);
    len_ = buf_.size();
    return GFSM_OK;
}

void FileBytes::close() {
    if (map_) munmap(map_, (size_t)len_);
    map_ = nullptr;
    buf_.clear();
    len_ = 0;
}

gfsm_status parse_text(const char *buf, uint64_t len, uint32_t rel_bits, HostGraph &g) {
    g = HostGraph();
    if (len < 6 || strncmp(buf, "t # 0\n", 6)) return GFSM_ERR_INVALID_DATA;  // :312-314
    // Header line (parseValues in header mode, :206-210): values 0 and 1 are
    // the vertex and edge-line counts.
    uint64_t pos = 6;
    uint32_t hv[4] = {0, 0, 0, 0};
    if (pos < len && buf[pos] == 't') {
        if (len - pos < 6 || strncmp(buf + pos, "t # -1", 6)) return GFSM_ERR_INVALID_DATA;
        return GFSM_OK;  // empty graph
    }
    const char *after = scan_values(buf + pos, buf + len, hv, 4);
    const uint32_t n = hv[0], ecount = hv[1];
    pos = (uint64_t)(after - buf);

    // Line-aligned chunks, scanned in parallel.
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    uint64_t body = len - pos;
    unsigned nt = (unsigned)std::min<uint64_t>(hw, std::max<uint64_t>(1, body / (1u << 20)));
    std::vector<uint64_t> cut(nt + 1);
    cut[0] = pos;
    cut[nt] = len;
    for (unsigned t = 1; t < nt; ++t) {
        uint64_t c = pos + body * t / nt;
        const char *nl = static_cast<const char *>(memchr(buf + c, '\n', len - c));
        c = nl ? (uint64_t)(nl - buf) + 1 : len;
        cut[t] = std::max(c, cut[t - 1]);
    }
    std::vector<ChunkOut> outs(nt);
    {
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t)
            th.emplace_back([&, t] { scan_chunk(buf, cut[t], cut[t + 1], len, outs[t]); });
        scan_chunk(buf, cut[0], cut[1], len, outs[0]);
        for (auto &x : th) x.join();
    }
    // Sequential semantics: the parse stops at the first 't' line or bad
    // line; a bad line (or a 'v' line inside the edge section, or a 't' line
    // other than "t # -1") before that point is ERR_INVALID_DATA.
    unsigned stop_chunk = nt;
    for (unsigned t = 0; t < nt; ++t)
        if (outs[t].first_stop != UINT64_MAX) { stop_chunk = t; break; }
    if (stop_chunk < nt && outs[stop_chunk].stop_kind == L_BAD) return GFSM_ERR_INVALID_DATA;
    unsigned last = stop_chunk < nt ? stop_chunk : nt - 1;
    bool seen_e = false;
    uint64_t nv = 0, ne = 0;
    for (unsigned t = 0; t <= last; ++t) {
        const ChunkOut &o = outs[t];
        if (o.first_v_after_e != UINT64_MAX) return GFSM_ERR_INVALID_DATA;
        if (seen_e && !o.vid.empty()) return GFSM_ERR_INVALID_DATA;
        if (!o.es.empty()) seen_e = true;
        nv += o.vid.size();
        ne += o.es.size();
    }
    // vertexSeen also counts the 'e' line that ends the vertex section (:344).
    uint64_t vseen = nv + (ne > 0 ? 1 : 0);
    if (vseen < n) return GFSM_ERR_MISSING_DATA;   // :347-349
    if (ne < ecount) return GFSM_ERR_MISSING_DATA; // :379-381

    g.n = n;
    g.vlabel.assign(n, 0);
    g.src.resize(ne);
    g.dst.resize(ne);
    g.lab.resize(ne);
    const uint32_t vert_bits = 32u - rel_bits;
    // each chunk's edges go to their place on its own thread; the vertex
    // lines are applied in file order (a repeated id keeps its last label)
    std::vector<uint64_t> eoff(last + 2, 0);
    for (unsigned t = 0; t <= last; ++t) eoff[t + 1] = eoff[t] + outs[t].es.size();
    std::atomic<bool> oob{false};
    auto place = [&](unsigned t) {
        const ChunkOut &o = outs[t];
        const uint64_t w0 = eoff[t];
        for (size_t i = 0; i < o.es.size(); ++i) {
            if (o.es[i] >= n || o.ed[i] >= n) {  // reference: out of bounds
                oob.store(true, std::memory_order_relaxed);
                return;
            }
            g.src[w0 + i] = o.es[i];
            g.dst[w0 + i] = o.ed[i];
            // (label << CCSRVertSize) keeps the low CCSRRelSize bits (:376)
            g.lab[w0 + i] = (uint8_t)(((uint32_t)(o.el[i] << vert_bits)) >> vert_bits);
        }
    };
    {
        std::vector<std::thread> th;
        for (unsigned t = 1; t <= last; ++t) th.emplace_back(place, t);
        place(0);
        for (unsigned t = 0; t <= last; ++t) {
            const ChunkOut &o = outs[t];
            for (size_t i = 0; i < o.vid.size(); ++i)
                if (o.vid[i] < n) g.vlabel[o.vid[i]] = o.vlab[i];
        }
        for (auto &x : th) x.join();
    }
    if (oob.load()) return GFSM_ERR_INVALID_DATA;
    return GFSM_OK;
}

// ---------------------------------------------------------------------------
// Planner
// ---------------------------------------------------------------------------
gfsm_status plan_query(const HostGraph &q, uint32_t rel_bits, Plan &p, const std::vector<double> *weight) {
    p = Plan();
    p.rel_bits = rel_bits;
    const uint32_t k = q.n;
    if (k == 0) return GFSM_ERR_QUERY;
    if (k > (uint32_t)MAXQ) return GFSM_ERR_TOO_LARGE;
    const size_t m = q.src.size();
    uint32_t deg[MAXQ] = {};
    for (uint32_t s : q.src) {
        if (s >= k) return GFSM_ERR_QUERY;
        deg[s]++;
    }
    for (uint32_t d : q.dst)
        if (d >= k) return GFSM_ERR_QUERY;
    for (uint32_t v = 0; v < k; ++v)
        if (!deg[v]) return GFSM_ERR_QUERY;  // no row: the reference walks past its CCSR
    // Query CCSR rows: degree descending, id ascending (HnHelper.cuh:26-31).
    uint32_t rowvid[MAXQ], rowidx[MAXQ];
    for (uint32_t v = 0; v < k; ++v) rowvid[v] = v;
    std::sort(rowvid, rowvid + k, [&](uint32_t a, uint32_t b) { return deg[a] != deg[b] ? deg[a] > deg[b] : a < b; });
    for (uint32_t i = 0; i < k; ++i) rowidx[rowvid[i]] = i;
    // row i = ent[rs[i], rs[i+1]): (target row, label) in input order, then
    // -- only if not in target order already -- sorted by target alone with
    // std::sort, the reference's steps (HnHelper.cuh:469-478): the order it
    // leaves entries of equal target in (their labels pick a requirement's
    // relation below) is the reference's own
    using Ent = std::pair<uint32_t, uint32_t>;
    uint32_t rs[MAXQ + 1] = {}, fill[MAXQ];
    for (uint32_t v = 0; v < k; ++v) rs[rowidx[v] + 1] = deg[v];
    for (uint32_t i = 0; i < k; ++i) rs[i + 1] += rs[i];
    std::copy(rs, rs + k, fill);
    std::vector<Ent> ent(m);
    for (size_t e = 0; e < m; ++e) ent[fill[rowidx[q.src[e]]]++] = {rowidx[q.dst[e]], q.lab[e]};
    uint32_t maxv = 0;
    auto by_target = [](const Ent &x, const Ent &y) { return x.first < y.first; };
    for (uint32_t i = 0; i < k; ++i) {
        Ent *b = ent.data() + rs[i], *e = ent.data() + rs[i + 1];
        if (!std::is_sorted(b, e, by_target)) std::sort(b, e, by_target);
        maxv = std::max(maxv, rs[i + 1] - rs[i]);
    }
    const Ent *E = ent.data();
    p.k = k;
    p.max_valency = maxv;
    p.order.assign(k, 0);
    p.header.assign(3 * (size_t)k, 0);
    p.reqs.assign(2 * (size_t)maxv * k, 0);
    // mapping[r]: -1 unseen, 0 seen (a neighbour of a placed row), d + 1 for
    // a row placed d depths ago.
    int32_t mapping[MAXQ];
    std::fill(mapping, mapping + k, -1);
    if (!weight) {
        mapping[0] = 0;  // HnGPU.cu:759-769: the first row has the maximal degree
    } else {
        // data-aware root: fewest data candidates per query edge
        uint32_t best = 0;
        double best_c = 0.0;
        for (uint32_t r = 0; r < k; ++r) {
            const double c = (*weight)[rowvid[r]] / (double)(rs[r + 1] - rs[r]);
            if (r == 0 || c < best_c) { best = r; best_c = c; }
        }
        mapping[best] = 0;
    }
    std::vector<Ent> rr;
    rr.reserve(maxv);
    for (uint32_t depth = 0; depth < k; ++depth) {  // HnGPU.cu:771-773
        uint32_t rel_depth = 0;
        bool found = false;
        if (!weight) {
            // ccsr.cpp:114-123: the first seen row in CCSR row order
            for (uint32_t i = 0; i < k; ++i) {
                if (mapping[i] == 0 && !found) {
                    mapping[i] = 1;
                    rel_depth = i;
                    found = true;
                } else if (mapping[i] > 0) {
                    mapping[i]++;
                }
            }
        } else {
            // data-aware: the seen row with the most placed neighbours (each
            // one a requirement that prunes), then the fewest data candidates
            uint32_t best_back = 0;
            double best_c = 0.0;
            for (uint32_t i = 0; i < k; ++i) {
                if (mapping[i] != 0) continue;
                uint32_t back = 0, last = ~0u;
                for (uint32_t x = rs[i]; x < rs[i + 1]; ++x)
                    if (E[x].first != last) {
                        last = E[x].first;
                        back += mapping[last] > 0 ? 1u : 0u;
                    }
                const double c = (*weight)[rowvid[i]];
                if (!found || back > best_back || (back == best_back && c < best_c)) {
                    rel_depth = i;
                    best_back = back;
                    best_c = c;
                    found = true;
                }
            }
            if (found)
                for (uint32_t i = 0; i < k; ++i) {
                    if (i == rel_depth) mapping[i] = 1;
                    else if (mapping[i] > 0) mapping[i]++;
                }
        }
        if (!found) return GFSM_ERR_QUERY;  // ccsr.cpp:126-128
        p.order[depth] = rel_depth;
        // ccsr.cpp:142-167
        rr.clear();
        for (uint32_t x = rs[rel_depth]; x < rs[rel_depth + 1]; ++x) {
            const uint32_t t = E[x].first;
            if (mapping[t] < 0) mapping[t] = 0;
            if (mapping[t] > 0) {
                uint32_t rel = E[x].second;
                for (uint32_t y = rs[t]; y < rs[t + 1]; ++y)
                    if (E[y].first == rel_depth) { rel = E[y].second; break; }
                rr.push_back({(uint32_t)(mapping[t] - 1), rel});
            }
        }
        // ccsr.cpp:169-196
        uint32_t firstq = 0, off = depth * maxv * 2;
        if (!rr.empty()) {
            std::sort(rr.begin(), rr.end(), by_target);  // by distance alone (ccsr.cpp:82-84, 170)
            p.reqs[off] = rr[0].first;
            p.reqs[off + 1] = rr[0].second;
            for (size_t i = 1; i < rr.size(); ++i) {
                p.reqs[off + 2 * i] = rr[i].first - rr[i - 1].first;
                p.reqs[off + 2 * i + 1] = rr[i].second;
            }
            firstq = p.reqs[off];
            for (size_t i = 0; i < rr.size(); ++i) {
                firstq = p.reqs[off + 2 * i];
                if (firstq) break;
            }
        }
        if ((firstq > depth && depth) || (depth && !firstq)) return GFSM_ERR_QUERY;
        p.header[depth * 3 + 0] = (uint32_t)rr.size();
        p.header[depth * 3 + 1] = off;
        p.header[depth * 3 + 2] = firstq;
    }
    for (size_t i = 0; i < (size_t)maxv * k; ++i)  // HnGPU.cu:807-813
        if (p.reqs[i * 2] > k) return GFSM_ERR_QUERY;

    // What the device plan needs beyond the reference tables.
    p.qvid.resize(k);
    p.qlabel.resize(k);
    p.qdeg.resize(k);
    for (uint32_t d = 0; d < k; ++d) {
        const uint32_t r = p.order[d], v = rowvid[r];
        p.qvid[d] = v;
        p.qlabel[d] = v < q.vlabel.size() ? q.vlabel[v] : 0;
        uint32_t nb = 0;  // distinct neighbour rows other than itself (k <= 32)
        for (uint32_t x = rs[r]; x < rs[r + 1]; ++x)
            if (E[x].first != r) nb |= 1u << E[x].first;
        p.qdeg[d] = (uint32_t)__builtin_popcount(nb);
    }
    // does row t hold (u, label)?  (any label when label < 0)
    auto holds = [&](uint32_t t, uint32_t u, int64_t label) {
        for (uint32_t y = rs[t]; y < rs[t + 1]; ++y)
            if (E[y].first == u && (label < 0 || E[y].second == (uint32_t)label)) return true;
        return false;
    };
    bool sym = true;
    for (uint32_t u = 0; u < k && sym; ++u)
        for (uint32_t x = rs[u]; x < rs[u + 1]; ++x)
            if (!holds(E[x].first, u, -1)) { sym = false; break; }
    p.symmetric = sym;
    // every entry has its reverse with the same label, and no (row, target)
    // pair repeats: a count that cannot depend on the matching order
    bool inv = sym;
    for (uint32_t u = 0; u < k && inv; ++u)
        for (uint32_t x = rs[u]; x < rs[u + 1] && inv; ++x) {
            if (x > rs[u] && E[x - 1].first == E[x].first) { inv = false; break; }
            inv = holds(E[x].first, u, E[x].second);
        }
    p.order_invariant = inv;
    p.planner = weight ? 1 : 0;
    return GFSM_OK;
}

// Symmetry breaking by a stabilizer chain (the conditions of Grochow and
// Kellis): with base points b_0, b_1, ... and G_0 = Aut(Q), G_{i+1} the
// stabilizer of b_i in G_i, the conditions f(b_i) < f(w) for every other w in
// b_i's G_i-orbit keep exactly one embedding of each orbit of Aut(Q) acting
// on embeddings (the action is free: embeddings are injective), and |Aut(Q)|
// is the product of the orbit sizes.  Orbits are found by searching for one
// automorphism per candidate image, never by listing the group.
void plan_symmetry(const HostGraph &q, Plan &p, bool vl) {
    p.aut = 1;
    p.sym_vl = vl;
    p.sym_cond.clear();
    const uint32_t k = q.n;
    if (!p.order_invariant || k < 2 || k > (uint32_t)MAXQ || p.qvid.size() != k) return;
    // edge label of each ordered pair (0: no edge; labels are >= 1 here or
    // the pair is absent), self-loops on the diagonal
    uint32_t lab[MAXQ * MAXQ] = {};
    for (size_t e = 0; e < q.src.size(); ++e) lab[(size_t)q.src[e] * k + q.dst[e]] = (uint32_t)q.lab[e] + 1u;
    uint32_t deg[MAXQ] = {}, vlab[MAXQ] = {};
    for (uint32_t a = 0; a < k; ++a) {
        for (uint32_t b = 0; b < k; ++b) deg[a] += lab[(size_t)a * k + b] != 0;
        vlab[a] = vl && a < q.vlabel.size() ? q.vlabel[a] : 0;
    }
    auto same_kind = [&](uint32_t a, uint32_t b) {
        return deg[a] == deg[b] && lab[(size_t)a * k + a] == lab[(size_t)b * k + b] && vlab[a] == vlab[b];
    };
    uint64_t budget = 1u << 22;  // search nodes over the whole analysis
    int32_t img[MAXQ], pre[MAXQ];
    uint32_t seq[MAXQ], nseq = 0;
    // extend the partial automorphism img along seq[i..nseq)
    auto extend = [&](auto &&self, uint32_t i) -> bool {
        if (i == nseq) return true;
        if (budget == 0) return false;
        --budget;
        const uint32_t a = seq[i];
        for (uint32_t w = 0; w < k; ++w) {
            if (pre[w] >= 0 || !same_kind(a, w)) continue;
            bool ok = true;
            for (uint32_t j = 0; j < i && ok; ++j) {
                const uint32_t x = seq[j], y = (uint32_t)img[x];
                ok = lab[(size_t)a * k + x] == lab[(size_t)w * k + y] && lab[(size_t)x * k + a] == lab[(size_t)y * k + w];
            }
            if (!ok) continue;
            img[a] = (int32_t)w;
            pre[w] = (int32_t)a;
            if (self(self, i + 1)) return true;
            img[a] = -1;
            pre[w] = -1;
        }
        return false;
    };
    uint32_t fixed[MAXQ], nfixed = 0, fixed_mask = 0;
    // is there an automorphism fixing fixed[0..nfixed) with a -> w?
    auto exists = [&](uint32_t a, uint32_t w) {
        std::fill(img, img + k, -1);
        std::fill(pre, pre + k, -1);
        for (uint32_t i = 0; i < nfixed; ++i) img[fixed[i]] = pre[fixed[i]] = (int32_t)fixed[i];
        if (pre[w] >= 0 || !same_kind(a, w)) return false;
        for (uint32_t i = 0; i < nfixed; ++i) {
            const uint32_t x = fixed[i];
            if (lab[(size_t)a * k + x] != lab[(size_t)w * k + x] || lab[(size_t)x * k + a] != lab[(size_t)x * k + w])
                return false;
        }
        img[a] = (int32_t)w;
        pre[w] = (int32_t)a;
        // the rest in matching order (neighbours of placed vertices first)
        nseq = 0;
        for (uint32_t i = 0; i < nfixed; ++i) seq[nseq++] = fixed[i];
        seq[nseq++] = a;
        for (uint32_t d = 0; d < k; ++d)
            if (img[p.qvid[d]] < 0) seq[nseq++] = p.qvid[d];
        return extend(extend, nfixed + 1);
    };
    uint64_t aut = 1;
    std::vector<std::pair<uint32_t, uint32_t>> cond;
    for (uint32_t d = 0; d < k; ++d) {
        const uint32_t b = p.qvid[d];
        uint64_t orbit = 1;
        for (uint32_t w = 0; w < k; ++w) {
            if (w == b || (fixed_mask >> w & 1u)) continue;
            if (exists(b, w)) {
                ++orbit;
                cond.push_back({b, w});
            }
            if (budget == 0) return;  // too large to analyse: no symmetry breaking
        }
        aut *= orbit;
        fixed[nfixed++] = b;
        fixed_mask |= 1u << b;
    }
    p.aut = aut;
    p.sym_cond = std::move(cond);
}

}  // namespace gfsm
