// Conversion of the reference BVH layouts into the compressed 8-wide layout.
//
// Input layouts (written by the reference adapters):
//   two-wide GPU nodes + 3-Vec4 triangles   src/imbatracer/core/gpu_adapter.cpp:62-143, 164-276
//   four-wide CPU nodes + 13-Vec4 packets   src/imbatracer/core/cpu_adapter.cpp:56-208, 229-365
//   instance nodes                          cpu_adapter.cpp:346-365 (shared by both)
// Bottom-level BVHs of all meshes and the top-level BVH share one node array; the scene root
// is the top-level root (scene.cpp:167-188), instance nodes point at mesh roots (`next`).
//
// The conversion parses the reachable tree into an intermediate binary/n-ary tree, splits
// leaves into runs of at most three primitives, collapses the tree into 8-wide nodes
// (repeatedly opening the child with the largest surface area), assigns child slots by
// direction octant and quantizes child boxes conservatively to 8 bits per plane.
// The node width is 8 or 4 (imbart_set_node_width): a 4-wide tree uses slots 0..3 of the
// same 80-byte record, ordered by the x/y quadrant, and leaves slots 4..7 empty.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <deque>
#include <unordered_map>
#include <vector>

#include "imbart_internal.h"

namespace imbart {

// Node width of the scenes converted from now on (IMBART_NODE_WIDTH, imbart_set_node_width).
namespace {
std::atomic<int> g_node_width{0};
}  // namespace

bool identity_instance(const WideInst& in) {
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 4; ++c)
            if (in.m[4 * a + c] != (a == c ? 1.0f : 0.0f)) return false;
    return true;
}

int current_node_width() {
    int w = g_node_width.load(std::memory_order_relaxed);
    if (w == 0) {
        const char* e = std::getenv("IMBART_NODE_WIDTH");
        const int v = e ? std::atoi(e) : 8;
        int expected = 0;
        g_node_width.compare_exchange_strong(expected, v == 4 ? 4 : 8);
        w = g_node_width.load(std::memory_order_relaxed);
    }
    return w;
}

namespace {

constexpr int kMaxLeafPrims = 3;
constexpr int kDummyRight = 0x76543210;
constexpr int kSentinel = (int)0x80000000;

struct IBox {
    float lo[3], hi[3];
    static IBox empty() {
        IBox b;
        for (int a = 0; a < 3; ++a) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; }
        return b;
    }
    void grow(const IBox& o) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], o.lo[a]); hi[a] = std::max(hi[a], o.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    void clip(const IBox& o) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::max(lo[a], o.lo[a]); hi[a] = std::min(hi[a], o.hi[a]); }
    }
    bool valid() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
    float half_area() const {
        float d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(hi[a] - lo[a], 0.0f);
        return d[0] * (d[1] + d[2]) + d[1] * d[2];
    }
};

// Intermediate tree node: internal (children) or leaf (a run of primitives).
struct INode {
    IBox box;
    std::vector<int> kids;
    int pbegin = 0, pcount = 0;  // leaf: indices into the tree's prim list
    bool leaf() const { return pcount > 0; }
};

struct ITree {
    std::vector<INode> nodes;
    std::vector<int> prims;   // leaf payload: triangle record index or instance record index
};

IBox box_from(const imbart_bbox& b) {
    IBox r;
    r.lo[0] = b.lo_x; r.lo[1] = b.lo_y; r.lo[2] = b.lo_z;
    r.hi[0] = b.hi_x; r.hi[1] = b.hi_y; r.hi[2] = b.hi_z;
    return r;
}

IBox tri_box(const WideTri& t) {
    IBox b = IBox::empty();
    b.grow(t.v0); b.grow(t.v1); b.grow(t.v2);
    return b;
}

// Appends a leaf over prims [first, first + n) of `tree.prims`, splitting runs longer than
// kMaxLeafPrims into a subtree ordered along the widest centroid axis. `prim_box(i)` gives
// the box of prim tree.prims[i]; chunk boxes are clipped to the reference leaf box, which
// keeps spatial-split (SBVH) references tight and is conservative for hits inside it.
template <typename PrimBox>
int add_leaf(ITree& tree, int first, int n, const IBox& leaf_box, PrimBox prim_box) {
    if (n <= kMaxLeafPrims) {
        INode nd;
        nd.box = leaf_box;
        nd.pbegin = first; nd.pcount = n;
        tree.nodes.push_back(nd);
        return (int)tree.nodes.size() - 1;
    }
    IBox cb = IBox::empty();
    for (int i = first; i < first + n; ++i) {
        IBox b = prim_box(tree.prims[i]);
        float c[3];
        for (int a = 0; a < 3; ++a) c[a] = 0.5f * (b.lo[a] + b.hi[a]);
        cb.grow(c);
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a) if (cb.hi[a] - cb.lo[a] > cb.hi[axis] - cb.lo[axis]) axis = a;
    std::stable_sort(tree.prims.begin() + first, tree.prims.begin() + first + n, [&](int x, int y) {
        IBox bx = prim_box(x), by = prim_box(y);
        return bx.lo[axis] + bx.hi[axis] < by.lo[axis] + by.hi[axis];
    });
    const int half = n / 2;
    IBox lb = IBox::empty(), rb = IBox::empty();
    for (int i = first; i < first + half; ++i) lb.grow(prim_box(tree.prims[i]));
    for (int i = first + half; i < first + n; ++i) rb.grow(prim_box(tree.prims[i]));
    lb.clip(leaf_box); rb.clip(leaf_box);
    if (!lb.valid()) lb = leaf_box;
    if (!rb.valid()) rb = leaf_box;
    const int l = add_leaf(tree, first, half, lb, prim_box);
    const int r = add_leaf(tree, first + half, n - half, rb, prim_box);
    INode nd;
    nd.box = leaf_box;
    nd.kids = {l, r};
    tree.nodes.push_back(nd);
    return (int)tree.nodes.size() - 1;
}

// ---------------------------------------------------------------------------------------
// Collapse into 8-wide nodes
// ---------------------------------------------------------------------------------------

struct WideBuilder {
    std::vector<WideNode>& out;
    int width;   // children per node: 8, or 4 (slots 0..3)
    WideBuilder(std::vector<WideNode>& o, int w) : out(o), width(w == 4 ? 4 : 8) {}

    // Children of a wide node: open the internal child with the largest area until `width`.
    static std::vector<int> gather(const ITree& t, int n, int width) {
        std::vector<int> kids;
        if (t.nodes[n].leaf()) { kids.push_back(n); return kids; }
        kids = t.nodes[n].kids;
        while ((int)kids.size() < width) {
            int best = -1; float best_area = -1.0f;
            for (int i = 0; i < (int)kids.size(); ++i) {
                const INode& k = t.nodes[kids[i]];
                if (k.leaf()) continue;
                if ((int)(kids.size() - 1 + k.kids.size()) > width) continue;
                const float a = k.box.half_area();
                if (a > best_area) { best_area = a; best = i; }
            }
            if (best < 0) break;
            const std::vector<int> sub = t.nodes[kids[best]].kids;
            kids.erase(kids.begin() + best);
            kids.insert(kids.end(), sub.begin(), sub.end());
        }
        return kids;
    }

    // Greedy slot assignment: slot s prefers children towards (s&1?+x:-x, s&2?+y:-y, s&4?+z:-z);
    // a 4-wide node uses slots 0..3, ordered by x and y alone.
    static void assign_slots(const ITree& t, const std::vector<int>& kids, int width, int slot_of[8]) {
        const int n = (int)kids.size();
        IBox all = IBox::empty();
        for (int k : kids) all.grow(t.nodes[k].box);
        float pc[3];
        for (int a = 0; a < 3; ++a) pc[a] = 0.5f * (all.lo[a] + all.hi[a]);
        struct Cand { float score; int kid, slot; };
        std::vector<Cand> cands;
        for (int i = 0; i < n; ++i) {
            const IBox& b = t.nodes[kids[i]].box;
            float d[3];
            for (int a = 0; a < 3; ++a) d[a] = 0.5f * (b.lo[a] + b.hi[a]) - pc[a];
            for (int s = 0; s < width; ++s) {
                const float score = (s & 1 ? d[0] : -d[0]) + (s & 2 ? d[1] : -d[1]) +
                                    (width == 4 ? 0.0f : (s & 4 ? d[2] : -d[2]));
                cands.push_back({score, i, s});
            }
        }
        std::stable_sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) { return x.score > y.score; });
        bool kid_done[8] = {}, slot_used[8] = {};
        for (int i = 0; i < 8; ++i) slot_of[i] = -1;
        for (const Cand& c : cands) {
            if (kid_done[c.kid] || slot_used[c.slot]) continue;
            kid_done[c.kid] = true; slot_used[c.slot] = true; slot_of[c.kid] = c.slot;
        }
    }

    // Quantizes one axis of up to 8 child boxes for the decoder used by the kernel:
    //     plane = P + (32768 + q) * 2^e,
    // where the GPU forms 32768 + q as a float with one byte permute (the byte in the mantissa
    // of 2^15) and evaluates the slab distance with a single FMA. The stored origin P lies
    // 32768 quanta below the node, so the slab terms carry an extra rounding of up to about
    // 2^-9 quanta; every child box is therefore enlarged by 1/128 of a quantum in addition to
    // the absolute pad (2^-20 of the node's magnitude). All checks here are exact (double).
    static void quantize_axis(const float* lo, const float* hi, const bool* valid, int nkids, float pad,
                              float* p_out, uint8_t* bexp_out, uint8_t* qlo, uint8_t* qhi) {
        double nlo = DBL_MAX, nhi = -DBL_MAX;
        for (int i = 0; i < nkids; ++i) {
            if (!valid[i]) continue;
            nlo = std::min(nlo, (double)lo[i] - pad);
            nhi = std::max(nhi, (double)hi[i] + pad);
        }
        if (nlo > nhi) { nlo = 0.0; nhi = 0.0; }
        const double ext = nhi - nlo;
        int e = -126;
        if (ext > 0.0) {
            int ex;
            std::frexp(ext / 252.0, &ex);   // ext / 252 < 2^ex; 3 quanta of slack for margins and P's rounding
            e = std::max(ex - 1, -126);
            while (e < 127 && std::ldexp(252.0, e) < ext) ++e;
        }
        float P = 0.0f;
        for (;;) {
            const double s = std::ldexp(1.0, e);
            const double margin = s / 128.0;
            const double origin = nlo - margin - 32768.0 * s;
            P = (float)origin;
            if ((double)P > origin) P = std::nextafter(P, -FLT_MAX);
            bool ok = true;
            for (int i = 0; i < nkids; ++i) {
                if (!valid[i]) { qlo[i] = 1; qhi[i] = 0; continue; }
                const double L = (double)lo[i] - pad - margin, H = (double)hi[i] + pad + margin;
                double ql = std::floor((L - (double)P) / s) - 32768.0;
                double qh = std::ceil((H - (double)P) / s) - 32768.0;
                while ((double)P + (32768.0 + ql) * s > L) ql -= 1;
                while ((double)P + (32768.0 + qh) * s < H) qh += 1;
                if (ql < 0 || qh > 255) { ok = false; break; }
                qlo[i] = (uint8_t)ql; qhi[i] = (uint8_t)qh;
            }
            if (ok || e >= 127) break;
            ++e;
        }
        *p_out = P;
        *bexp_out = (uint8_t)(e + 127);
    }

    // Builds the wide tree of `t` rooted at intermediate node `root`. Leaf primitives are
    // appended through `emit(prim)` which returns the index of the emitted record.
    template <typename Emit>
    int build(const ITree& t, int root, Emit emit) {
        const int wroot = (int)out.size();
        out.emplace_back();
        std::deque<std::pair<int, int>> work;
        work.push_back({wroot, root});
        while (!work.empty()) {
            auto [w, n] = work.front();
            work.pop_front();
            std::vector<int> kids = gather(t, n, width);
            int slot_of[8];
            assign_slots(t, kids, width, slot_of);
            int kid_in_slot[8];
            for (int s = 0; s < 8; ++s) kid_in_slot[s] = -1;
            for (int i = 0; i < (int)kids.size(); ++i) kid_in_slot[slot_of[i]] = kids[i];

            WideNode nd;
            std::memset(&nd, 0, sizeof(nd));
            // Internal children are allocated contiguously in slot order.
            int n_internal = 0;
            for (int s = 0; s < 8; ++s)
                if (kid_in_slot[s] >= 0 && !t.nodes[kid_in_slot[s]].leaf()) nd.imask |= (uint8_t)(1u << s), ++n_internal;
            const int child_base = (int)out.size();
            out.resize(out.size() + n_internal);
            nd.child_base = (uint32_t)child_base;
            int prim_base = -1, prim_off = 0;
            int rank = 0;
            for (int s = 0; s < 8; ++s) {
                const int k = kid_in_slot[s];
                if (k < 0) continue;
                const INode& kn = t.nodes[k];
                if (!kn.leaf()) {
                    work.push_back({child_base + rank, k});
                    ++rank;
                    continue;
                }
                for (int j = 0; j < kn.pcount; ++j) {
                    const int rec = emit(t.prims[kn.pbegin + j]);
                    if (prim_base < 0) prim_base = rec;
                }
                nd.meta[s] = (uint8_t)((kn.pcount << 5) | prim_off);
                prim_off += kn.pcount;
            }
            nd.prim_base = (uint32_t)(prim_base < 0 ? 0 : prim_base);

            // Quantize the child boxes.
            float lo[3][8], hi[3][8];
            bool valid[8];
            float mag = 0.0f;
            for (int s = 0; s < 8; ++s) {
                valid[s] = kid_in_slot[s] >= 0;
                for (int a = 0; a < 3; ++a) { lo[a][s] = 0.0f; hi[a][s] = 0.0f; }
                if (!valid[s]) continue;
                const IBox& b = t.nodes[kid_in_slot[s]].box;
                for (int a = 0; a < 3; ++a) {
                    lo[a][s] = b.lo[a]; hi[a][s] = b.hi[a];
                    mag = std::max(mag, std::max(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
                    mag = std::max(mag, b.hi[a] - b.lo[a]);
                }
            }
            const float pad = mag * 9.5367431640625e-07f + 1e-30f;  // 2^-20 of the node's scale
            uint8_t bexp[3];
            float p[3];
            quantize_axis(lo[0], hi[0], valid, 8, pad, &p[0], &bexp[0], nd.qlo_x, nd.qhi_x);
            quantize_axis(lo[1], hi[1], valid, 8, pad, &p[1], &bexp[1], nd.qlo_y, nd.qhi_y);
            quantize_axis(lo[2], hi[2], valid, 8, pad, &p[2], &bexp[2], nd.qlo_z, nd.qhi_z);
            nd.px = p[0]; nd.py = p[1]; nd.pz = p[2];
            nd.ex = bexp[0]; nd.ey = bexp[1]; nd.ez = bexp[2];
            out[w] = nd;
        }
        return wroot;
    }
};

// ---------------------------------------------------------------------------------------
// Reference layout parsing
// ---------------------------------------------------------------------------------------

struct Parser {
    HostWideScene& out;
    std::string err;
    explicit Parser(HostWideScene& o) : out(o) {}

    // Parses a bottom-level triangle run of the two-wide layout starting at Vec4 index `at`.
    bool tri_run2(const imbart_vec4* tris, int n_vec4, int at, std::vector<int>& recs) {
        for (int guard = 0;; ++guard) {
            if (at < 0 || at + 3 > n_vec4 || guard > (1 << 26)) { err = "triangle run out of bounds"; return false; }
            WideTri t;
            std::memset(&t, 0, sizeof(t));
            t.v0[0] = tris[at].x; t.v0[1] = tris[at].y; t.v0[2] = tris[at].z;
            t.v1[0] = tris[at + 1].x; t.v1[1] = tris[at + 1].y; t.v1[2] = tris[at + 1].z;
            t.v2[0] = tris[at + 2].x; t.v2[1] = tris[at + 2].y; t.v2[2] = tris[at + 2].z;
            t.id = float_bits(tris[at + 1].w);
            recs.push_back((int)out.tris.size());
            out.tris.push_back(t);
            const bool last = float_bits(tris[at + 2].w) == kSentinel;
            at += 3;
            if (last) return true;
        }
    }

    // Parses a bottom-level packet run of the four-wide layout starting at Vec4 index `at`.
    bool tri_run4(const imbart_vec4* tris, int n_vec4, int at, std::vector<int>& recs) {
        for (int guard = 0;; ++guard) {
            if (at < 0 || at >= n_vec4 || guard > (1 << 24)) { err = "triangle packet run out of bounds"; return false; }
            const imbart_vec4& s = tris[at];
            if (float_bits(s.x) == kSentinel && float_bits(s.y) == kSentinel &&
                float_bits(s.z) == kSentinel && float_bits(s.w) == kSentinel)
                return true;
            if (at + 13 > n_vec4) { err = "triangle packet out of bounds"; return false; }
            const float* raw = &tris[at].x;
            for (int j = 0; j < 4; ++j) {
                const int id = float_bits(raw[48 + j]);
                if (id == kSentinel) continue;
                WideTri t;
                std::memset(&t, 0, sizeof(t));
                for (int a = 0; a < 3; ++a) {
                    const float v0 = raw[4 * a + j];
                    const float e1 = raw[12 + 4 * a + j];
                    const float e2 = raw[24 + 4 * a + j];
                    t.v0[a] = v0;
                    t.v1[a] = v0 - e1;   // e1 = v0 - v1 (cpu_adapter.cpp:138)
                    t.v2[a] = v0 + e2;   // e2 = v2 - v0 (cpu_adapter.cpp:139)
                }
                t.id = id;
                recs.push_back((int)out.tris.size());
                out.tris.push_back(t);
            }
            at += 13;
        }
    }

    // Generic recursive parse. `Kids(node, cb)` enumerates (code, box) children of a node;
    // `Run(code, recs)` parses a leaf payload run into record indices.
    template <typename Kids, typename Run, typename PrimBox>
    int parse(ITree& tree, int node, int n_nodes, const IBox& box, int depth, Kids kids, Run run, PrimBox pbox) {
        if (node < 0 || node >= n_nodes) { err = "node index out of bounds"; return -1; }
        if (depth > 4096) { err = "BVH deeper than 4096 levels"; return -1; }
        std::vector<std::pair<int, IBox>> ch;
        kids(node, ch);
        std::vector<int> parsed;
        for (auto& [code, cbox] : ch) {
            if (code >= 0) {
                const int k = parse(tree, code, n_nodes, cbox, depth + 1, kids, run, pbox);
                if (k < 0) return -1;
                parsed.push_back(k);
            } else {
                std::vector<int> recs;
                if (!run(~code, recs)) return -1;
                if (recs.empty()) continue;
                const int first = (int)tree.prims.size();
                tree.prims.insert(tree.prims.end(), recs.begin(), recs.end());
                parsed.push_back(add_leaf(tree, first, (int)recs.size(), cbox, pbox));
            }
        }
        if (parsed.empty()) { err = "BVH node without children"; return -1; }
        if (parsed.size() == 1) return parsed[0];   // single-leaf wrapper
        INode nd;
        nd.box = box;
        nd.kids = parsed;
        tree.nodes.push_back(nd);
        return (int)tree.nodes.size() - 1;
    }
};

// Shared driver: parses the top level, converts each distinct mesh BVH once, then the top level.
template <typename Kids, typename BottomRun>
std::string convert_common(int root, int n_nodes, const imbart_instance_node* insts, int n_insts,
                           HostWideScene& out, Kids kids, BottomRun bottom_run, int node_width) {
    if (node_width < 0) node_width = current_node_width();
    if (node_width != 4 && node_width != 8) return "node width must be 4 or 8";
    out.nodes.clear(); out.tris.clear(); out.insts.clear();
    out.node_width = node_width;
    Parser ps(out);
    if (root < 0 || root >= n_nodes) return "root out of bounds";

    // Top level: leaves are runs of instance nodes closed by pad[0] == -1.
    std::vector<int> inst_src;  // instance-record index -> source instance node index
    auto inst_run = [&](int at, std::vector<int>& recs) -> bool {
        for (int guard = 0;; ++guard) {
            if (at < 0 || at >= n_insts || guard > n_insts) { ps.err = "instance run out of bounds"; return false; }
            recs.push_back((int)inst_src.size());
            inst_src.push_back(at);
            if (insts[at].pad[0] == -1) return true;
            ++at;
        }
    };
    ITree top;
    IBox root_box = IBox::empty();
    {
        std::vector<std::pair<int, IBox>> ch;
        kids(root, ch);
        for (auto& c : ch) root_box.grow(c.second);
    }
    auto top_pbox = [&](int) { return root_box; };  // refined below per leaf via clip
    const int top_root = ps.parse(top, root, n_nodes, root_box, 0, kids, inst_run, top_pbox);
    if (top_root < 0) return ps.err;

    // Bottom level: one wide tree per distinct mesh root.
    std::unordered_map<int, int> wide_root_of;
    WideBuilder wb(out.nodes, node_width);
    for (int src : inst_src) {
        const int mroot = insts[src].next;
        if (wide_root_of.count(mroot)) continue;
        if (mroot < 0 || mroot >= n_nodes) return "instance mesh root out of bounds";
        ITree bt;
        std::vector<std::pair<int, IBox>> ch;
        kids(mroot, ch);
        IBox mbox = IBox::empty();
        for (auto& c : ch) mbox.grow(c.second);
        auto tri_pbox = [&](int rec) { return tri_box(out.tris[rec]); };
        // Triangle records are emitted by the run parser into out.tris; the wide builder
        // then re-emits them in leaf order.
        const int tris_before = (int)out.tris.size();
        auto run = [&](int at, std::vector<int>& recs) { return bottom_run(ps, at, recs); };
        const int br = ps.parse(bt, mroot, n_nodes, mbox, 0, kids, run, tri_pbox);
        if (br < 0) return ps.err;
        std::vector<WideTri> parsed(out.tris.begin() + tris_before, out.tris.end());
        out.tris.resize(tris_before);
        auto emit_tri = [&](int rec) {
            out.tris.push_back(parsed[rec - tris_before]);
            return (int)out.tris.size() - 1;
        };
        wide_root_of[mroot] = wb.build(bt, br, emit_tri);
    }

    // Top level.
    const int top_first = (int)out.nodes.size();
    auto emit_inst = [&](int rec) {
        const imbart_instance_node& in = insts[inst_src[rec]];
        WideInst wi;
        std::memset(&wi, 0, sizeof(wi));
        std::memcpy(wi.m, in.transf, sizeof(wi.m));
        wi.id = in.id;
        wi.root = wide_root_of[in.next];
        out.insts.push_back(wi);
        return (int)out.insts.size() - 1;
    };
    out.root = wb.build(top, top_root, emit_inst);
    out.top_nodes = (int)out.nodes.size() - top_first;
    if (out.nodes.size() >= (size_t)1 << 30 || out.tris.size() >= (size_t)1 << 30 ||
        out.insts.size() >= (size_t)1 << 30)
        return "scene too large for 30-bit indices";
    return "";
}

}  // namespace

std::string convert_node2(int root, const imbart_node2* nodes, int n_nodes,
                          const imbart_instance_node* insts, int n_insts,
                          const imbart_vec4* tris, int n_tri_vec4, HostWideScene& out, int node_width) {
    auto kids = [&](int n, std::vector<std::pair<int, IBox>>& ch) {
        const imbart_node2& nd = nodes[n];
        ch.push_back({nd.left, box_from(nd.left_bb)});
        if (nd.right != kDummyRight) ch.push_back({nd.right, box_from(nd.right_bb)});
    };
    auto bottom_run = [&](Parser& ps, int at, std::vector<int>& recs) {
        return ps.tri_run2(tris, n_tri_vec4, at, recs);
    };
    return convert_common(root, n_nodes, insts, n_insts, out, kids, bottom_run, node_width);
}

std::string convert_node4(int root, const imbart_node4* nodes, int n_nodes,
                          const imbart_instance_node* insts, int n_insts,
                          const imbart_vec4* tris, int n_tri_vec4, HostWideScene& out, int node_width) {
    auto kids = [&](int n, std::vector<std::pair<int, IBox>>& ch) {
        const imbart_node4& nd = nodes[n];
        for (int j = 0; j < 4; ++j) {
            if (nd.children[j] == 0) continue;
            IBox b;
            b.lo[0] = nd.min_x[j]; b.lo[1] = nd.min_y[j]; b.lo[2] = nd.min_z[j];
            b.hi[0] = nd.max_x[j]; b.hi[1] = nd.max_y[j]; b.hi[2] = nd.max_z[j];
            ch.push_back({nd.children[j], b});
        }
    };
    auto bottom_run = [&](Parser& ps, int at, std::vector<int>& recs) {
        return ps.tri_run4(tris, n_tri_vec4, at, recs);
    };
    return convert_common(root, n_nodes, insts, n_insts, out, kids, bottom_run, node_width);
}

}  // namespace imbart

extern "C" int imbart_set_node_width(int width) {
    if (width != 4 && width != 8) {
        imbart::set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_set_node_width: width must be 4 or 8");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    imbart::current_node_width();   // settle the environment default first
    imbart::g_node_width.store(width, std::memory_order_relaxed);
    return 0;
}

extern "C" int imbart_get_node_width(void) { return imbart::current_node_width(); }

extern "C" int imbart_wide_from_node2(int root, const imbart_node2* nodes, int n_nodes,
                                      const imbart_instance_node* instances, int n_instances,
                                      const imbart_vec4* tris, int n_tri_vec4,
                                      void* nodes_out, int nodes_cap, void* tris_out, int tris_cap,
                                      void* insts_out, int insts_cap, int* counts) {
    using namespace imbart;
    if (!nodes || !instances || !tris || !counts) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_wide_from_node2: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    HostWideScene h;
    const std::string err = convert_node2(root, nodes, n_nodes, instances, n_instances, tris, n_tri_vec4, h);
    if (!err.empty()) {
        set_error(IMBART_ERR_BAD_SCENE, "imbart_wide_from_node2: " + err);
        return IMBART_ERR_BAD_SCENE;
    }
    counts[0] = (int)h.nodes.size();
    counts[1] = (int)h.tris.size();
    counts[2] = (int)h.insts.size();
    counts[3] = h.root;
    if (nodes_out && nodes_cap > 0)
        std::memcpy(nodes_out, h.nodes.data(), sizeof(WideNode) * std::min<size_t>(nodes_cap, h.nodes.size()));
    if (tris_out && tris_cap > 0)
        std::memcpy(tris_out, h.tris.data(), sizeof(WideTri) * std::min<size_t>(tris_cap, h.tris.size()));
    if (insts_out && insts_cap > 0)
        std::memcpy(insts_out, h.insts.data(), sizeof(WideInst) * std::min<size_t>(insts_cap, h.insts.size()));
    return 0;
}

namespace imbart {

void attach_masks(HostWideScene& out, const int* indices, int n_indices,
                  const imbart_vec2* texcoords, int n_texcoords,
                  const imbart_mask_desc* masks, int n_masks,
                  const char* mask_buffer, int mask_buffer_size) {
    out.masked = false;
    if (!indices || !masks || !mask_buffer || n_masks <= 0) return;
    // The default descriptor is a 1x1 opaque texel at offset 0 (mask.h:13-15, 31-34).
    bool any = false;
    for (int i = 0; i < n_masks && !any; ++i) {
        const imbart_mask_desc& d = masks[i];
        if (d.width * d.height != 1) { any = true; break; }
        if (d.offset < 0 || d.offset >= mask_buffer_size || mask_buffer[d.offset] == 0) any = true;
    }
    if (!any) return;
    out.masked = true;
    out.indices.assign(indices, indices + n_indices);
    if (texcoords && n_texcoords > 0) out.texcoords.assign(texcoords, texcoords + n_texcoords);
    out.masks.assign(masks, masks + n_masks);
    out.mask_buffer.assign((const uint8_t*)mask_buffer, (const uint8_t*)mask_buffer + mask_buffer_size);
}

}  // namespace imbart
