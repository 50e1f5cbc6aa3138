// Geometry image of the walk: the triangles of all surfaces and a threaded (stackless) BVH over
// them, laid out for coalesced 16-byte loads on the GPU.
//
// Triangles: the reference stores surfaces as FP64 vertex arrays plus int3 index arrays and its
// BVH leaves as (surfId, trIndex) indirections (mcml_types.h:31-37, mcml_intersection.h:24-28).
// Here every triangle becomes one 48-byte record {v0.xyz, surf}, {v1.xyz, global id}, {v2.xyz, band}
// (band: width of the FP64 edge re-test band, see geom.cuh)
// of FP32 vertices, stored in leaf order so a leaf's triangles are contiguous.
//
// Nodes: 32 bytes {lo.xyz, child}, {hi.xyz, miss}. child >= 0 is the first child of an inner
// node (its sibling is reached through the first child's miss link); child < 0 encodes a leaf as
// -1 - (first_triangle << 3 | (count - 1)). miss is the node to visit when this node's box is
// missed or its subtree is done (-1 ends the traversal). The first nodes in breadth-first order
// come first in the array so the top levels can be staged in shared memory.
//
// The tree is either the caller's prebuilt reference BVH (input->bvhTree, the output of the
// reference's GenerateBVHTree, mcml_intersection.cpp:316-344, which the reference's launcher
// builds before LaunchOMP, launcher_mpi.cpp:396) converted node for node, or a binned-SAH tree
// built here. Node boxes are always recomputed from the FP32 vertices and padded so the FP32 slab
// test never culls a triangle that the FP32/FP64 triangle test would hit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>

#include "xmc_internal.h"

namespace xmc {
namespace {

struct BNode {
    float lo[3], hi[3];
    int left = -1, right = -1;  // inner node children
    int first = 0, count = 0;   // leaf: triangles [first, first + count) of `order`
};

struct Builder {
    std::vector<float> v;       // 9 floats per triangle (v0, v1, v2)
    std::vector<int> surf;      // surface of each triangle
    std::vector<int> order;     // triangle permutation (leaf order)
    std::vector<BNode> nodes;
    std::vector<float> cen;     // 3 floats per triangle

    void tri_box(int t, float lo[3], float hi[3]) const {
        const float* p = &v[9 * (size_t)t];
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(p[k], std::min(p[3 + k], p[6 + k]));
            hi[k] = std::max(p[k], std::max(p[3 + k], p[6 + k]));
        }
    }

    void range_box(int b, int e, float lo[3], float hi[3]) const {
        for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
        for (int i = b; i < e; ++i) {
            float l[3], h[3];
            tri_box(order[i], l, h);
            for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], l[k]); hi[k] = std::max(hi[k], h[k]); }
        }
    }

    static float area(const float lo[3], const float hi[3]) {
        float dx = std::max(0.f, hi[0] - lo[0]), dy = std::max(0.f, hi[1] - lo[1]), dz = std::max(0.f, hi[2] - lo[2]);
        return dx * dy + dy * dz + dz * dx;
    }

    int make_leaf(int b, int e) {
        BNode n;
        range_box(b, e, n.lo, n.hi);
        n.first = b;
        n.count = e - b;
        nodes.push_back(n);
        return (int)nodes.size() - 1;
    }

    // Leaves hold at most 8 triangles (3-bit count); a longer run becomes a small subtree.
    int make_leaves(int b, int e) {
        if (e - b <= 8) return make_leaf(b, e);
        int m = b + (e - b) / 2;
        int l = make_leaves(b, m), r = make_leaves(m, e);
        return make_inner(l, r);
    }

    int make_inner(int l, int r) {
        BNode n;
        for (int k = 0; k < 3; ++k) {
            n.lo[k] = std::min(nodes[l].lo[k], nodes[r].lo[k]);
            n.hi[k] = std::max(nodes[l].hi[k], nodes[r].hi[k]);
        }
        n.left = l;
        n.right = r;
        nodes.push_back(n);
        return (int)nodes.size() - 1;
    }

    // Binned SAH (16 bins per axis over the centroid bounds), leaves of <= 4 triangles.
    int build_sah(int b, int e, int depth) {
        int count = e - b;
        if (count <= 4 || depth > 48) return make_leaves(b, e);
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int i = b; i < e; ++i)
            for (int k = 0; k < 3; ++k) {
                float c = cen[3 * (size_t)order[i] + k];
                clo[k] = std::min(clo[k], c);
                chi[k] = std::max(chi[k], c);
            }
        const int NB = 16;
        float best_cost = INFINITY;
        int best_axis = -1, best_split = 0;
        for (int k = 0; k < 3; ++k) {
            float ext = chi[k] - clo[k];
            if (!(ext > 0.f)) continue;
            int cnt[NB] = {0};
            float blo[NB][3], bhi[NB][3];
            for (int j = 0; j < NB; ++j)
                for (int a = 0; a < 3; ++a) { blo[j][a] = INFINITY; bhi[j][a] = -INFINITY; }
            float scale = NB / ext;
            for (int i = b; i < e; ++i) {
                int t = order[i];
                int j = std::min(NB - 1, (int)((cen[3 * (size_t)t + k] - clo[k]) * scale));
                cnt[j]++;
                float l[3], h[3];
                tri_box(t, l, h);
                for (int a = 0; a < 3; ++a) { blo[j][a] = std::min(blo[j][a], l[a]); bhi[j][a] = std::max(bhi[j][a], h[a]); }
            }
            float rlo[NB][3], rhi[NB][3];
            int rcnt[NB];
            float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
            int acc = 0;
            for (int j = NB - 1; j > 0; --j) {
                acc += cnt[j];
                for (int a = 0; a < 3; ++a) { alo[a] = std::min(alo[a], blo[j][a]); ahi[a] = std::max(ahi[a], bhi[j][a]); }
                rcnt[j] = acc;
                for (int a = 0; a < 3; ++a) { rlo[j][a] = alo[a]; rhi[j][a] = ahi[a]; }
            }
            float llo[3] = {INFINITY, INFINITY, INFINITY}, lhi[3] = {-INFINITY, -INFINITY, -INFINITY};
            int lc = 0;
            for (int j = 1; j < NB; ++j) {
                lc += cnt[j - 1];
                for (int a = 0; a < 3; ++a) { llo[a] = std::min(llo[a], blo[j - 1][a]); lhi[a] = std::max(lhi[a], bhi[j - 1][a]); }
                if (lc == 0 || rcnt[j] == 0) continue;
                float c = area(llo, lhi) * lc + area(rlo[j], rhi[j]) * rcnt[j];
                if (c < best_cost) { best_cost = c; best_axis = k; best_split = j; }
            }
        }
        int mid;
        if (best_axis < 0) {
            mid = b + count / 2;  // all centroids equal: split by count
        } else {
            float lo[3], hi[3];
            range_box(b, e, lo, hi);
            float leaf_cost = area(lo, hi) * count;
            if (count <= 8 && leaf_cost <= best_cost + area(lo, hi) * 1.0f) return make_leaf(b, e);
            int k = best_axis;
            float scale = NB / (chi[k] - clo[k]);
            auto it = std::stable_partition(order.begin() + b, order.begin() + e, [&](int t) {
                return std::min(NB - 1, (int)((cen[3 * (size_t)t + k] - clo[k]) * scale)) < best_split;
            });
            mid = (int)(it - order.begin());
            if (mid == b || mid == e) mid = b + count / 2;
        }
        int l = build_sah(b, mid, depth + 1);
        int r = build_sah(mid, e, depth + 1);
        return make_inner(l, r);
    }
};

// host threads for a loop over n independent items: one below 65,536 items, else up to 16
static unsigned host_parts(size_t n) {
    return n < 65536 ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
}

void pad_box(float lo[3], float hi[3]) {
    for (int k = 0; k < 3; ++k) {
        float m = 4e-7f * std::max(1.0f, std::max(std::fabs(lo[k]), std::fabs(hi[k])));
        lo[k] -= m;
        hi[k] += m;
    }
}

}  // namespace

bool build_geometry(const InputInfo* in, GeomImage* out, std::string* err, int gpu_device) {
    Builder B;
    int ntri = 0;
    std::vector<int> surf_base(in->numberOfSurfaces + 1, 0);
    for (int s = 0; s < in->numberOfSurfaces; ++s) {
        const Surface& S = in->surface[s];
        if (S.numberOfTriangles < 0 || S.numberOfVertices < 0) { *err = "surface " + std::to_string(s) + ": negative counts"; return false; }
        if (S.numberOfTriangles > 0 && (!S.triangles || !S.vertices)) { *err = "surface " + std::to_string(s) + ": null arrays"; return false; }
        surf_base[s] = ntri;
        ntri += S.numberOfTriangles;
    }
    surf_base[in->numberOfSurfaces] = ntri;
    if (ntri >= (1 << 27)) { *err = "too many triangles"; return false; }
    B.v.resize(9 * (size_t)ntri);
    B.surf.resize(ntri);
    B.cen.resize(3 * (size_t)ntri);
    // FP32 vertices, centroids and surface ids, each host thread a range of triangles; a bad vertex
    // index is reported for the first triangle (in input order) that has one
    const unsigned parts = host_parts(ntri);
    const size_t per = ((size_t)ntri + parts - 1) / parts;
    std::vector<int> bad(parts, -1);
    parallel_parts(parts, [&](unsigned part) {
        const int t0 = (int)std::min((size_t)ntri, part * per), t1 = (int)std::min((size_t)ntri, (part + 1) * per);
        int s = (int)(std::upper_bound(surf_base.begin(), surf_base.end() - 1, t0) - surf_base.begin()) - 1;
        for (int t = t0; t < t1; ++t) {
            while (t >= surf_base[s + 1]) ++s;
            const Surface& S = in->surface[s];
            const xmc_ref_int3& T = S.triangles[t - surf_base[s]];
            const int id[3] = {T.x, T.y, T.z};
            for (int c = 0; c < 3; ++c) {
                if (id[c] < 0 || id[c] >= S.numberOfVertices) {
                    bad[part] = t;
                    return;
                }
                const xmc_ref_double3& P = S.vertices[id[c]];
                B.v[9 * (size_t)t + 3 * c + 0] = (float)P.x;
                B.v[9 * (size_t)t + 3 * c + 1] = (float)P.y;
                B.v[9 * (size_t)t + 3 * c + 2] = (float)P.z;
            }
            for (int k = 0; k < 3; ++k)
                B.cen[3 * (size_t)t + k] = (B.v[9 * (size_t)t + k] + B.v[9 * (size_t)t + 3 + k] + B.v[9 * (size_t)t + 6 + k]) / 3.0f;
            B.surf[t] = s;
        }
    });
    for (unsigned part = 0; part < parts; ++part)
        if (bad[part] >= 0) {
            const int t = bad[part];
            const int s = (int)(std::upper_bound(surf_base.begin(), surf_base.end() - 1, t) - surf_base.begin()) - 1;
            *err = "surface " + std::to_string(s) + " triangle " + std::to_string(t - surf_base[s]) +
                   ": vertex index out of range";
            return false;
        }
    out->nodes.clear();
    out->tris.clear();
    out->n_nodes = out->n_tris = 0;
    if (ntri == 0) return true;

    int root = -1;
    const BVHTree* ref = in->bvhTree;
    bool use_ref = ref && ref->nodes && ref->numOfNodes > 0 && ref->triangles && ref->numOfTriangles == ntri &&
                   ref->root >= 0 && ref->root < ref->numOfNodes;
    if (use_ref) {
        // Convert the reference tree: leaves keep their triangle runs, inner nodes their children.
        B.order.clear();
        B.order.reserve(ntri);
        std::function<int(int, int)> conv = [&](int ni, int depth) -> int {
            if (ni < 0 || ni >= ref->numOfNodes || depth > 200) return -2;
            const BVHNode& N = ref->nodes[ni];
            if (N.offset >= 0) {
                if (N.numOfTriangles <= 0 || N.offset + N.numOfTriangles > ref->numOfTriangles) return -2;
                int b = (int)B.order.size();
                for (int i = 0; i < N.numOfTriangles; ++i) {
                    const Triangle& T = ref->triangles[N.offset + i];
                    if (T.surfId < 0 || T.surfId >= in->numberOfSurfaces ||
                        T.trIndex < 0 || T.trIndex >= in->surface[T.surfId].numberOfTriangles) return -2;
                    B.order.push_back(surf_base[T.surfId] + T.trIndex);
                }
                return B.make_leaves(b, (int)B.order.size());
            }
            int l = conv(N.leftNode, depth + 1);
            if (l < 0) return -2;
            int r = conv(N.rightNode, depth + 1);
            if (r < 0) return -2;
            return B.make_inner(l, r);
        };
        root = conv(ref->root, 0);
        if (root < 0 || (int)B.order.size() != ntri) {
            // Not a usable tree (inconsistent indices): build our own instead.
            use_ref = false;
            B.nodes.clear();
        }
    }
    if (!use_ref && gpu_device >= 0 && ntri >= 2) {
        // Linear BVH topology from the GPU over the ordinary triangles. Triangles far larger than the
        // median (the planes of a layer stack) would sit in deep leaves with scene-sized boxes under a
        // spatial-median split, so they get their own binned-SAH subtree beside it, at the root.
        std::vector<float> ext(ntri);
        for (int t = 0; t < ntri; ++t) {
            float lo[3], hi[3];
            B.tri_box(t, lo, hi);
            ext[t] = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
        }
        std::vector<float> sorted_ext(ext);
        std::nth_element(sorted_ext.begin(), sorted_ext.begin() + ntri / 2, sorted_ext.end());
        const float big = 16.0f * sorted_ext[ntri / 2];
        std::vector<int> small, large;
        for (int t = 0; t < ntri; ++t) (big > 0.0f && ext[t] > big ? large : small).push_back(t);
        const int ns = (int)small.size();
        B.order.clear();
        int root_s = -1;
        if (ns >= 2) {
            std::vector<float> cen_s(3 * (size_t)ns);
            for (int i = 0; i < ns; ++i)
                for (int k = 0; k < 3; ++k) cen_s[3 * (size_t)i + k] = B.cen[3 * (size_t)small[i] + k];
            std::vector<int> order_s;
            std::vector<int2> child, range;
            if (!gpu_lbvh_topology(cen_s, ns, gpu_device, &order_s, &child, &range, err)) return false;
            B.order.resize(ns);
            for (int i = 0; i < ns; ++i) B.order[i] = small[order_s[i]];
            B.nodes.reserve(2 * (size_t)ntri);
            // post-order over the internal nodes with an explicit stack: (node, children done);
            // subtrees of <= 4 triangles (contiguous in the sorted order) become leaves
            std::vector<int> built(ns - 1, -1);
            std::vector<std::pair<int, bool>> st{{0, false}};
            auto leaf_of = [&](int c) { return B.make_leaf(-1 - c, -c); };
            while (!st.empty()) {
                auto [x, done] = st.back();
                st.pop_back();
                const int2 rg = range[x];
                if (rg.y - rg.x + 1 <= 4) {
                    built[x] = B.make_leaf(rg.x, rg.y + 1);
                    continue;
                }
                const int2 c = child[x];
                if (!done) {
                    st.push_back({x, true});
                    if (c.y >= 0) st.push_back({c.y, false});
                    if (c.x >= 0) st.push_back({c.x, false});
                    continue;
                }
                const int l = c.x >= 0 ? built[c.x] : leaf_of(c.x);
                const int r = c.y >= 0 ? built[c.y] : leaf_of(c.y);
                built[x] = B.make_inner(l, r);
            }
            root_s = built[0];
        } else if (ns == 1) {
            B.order.push_back(small[0]);
            root_s = B.make_leaf(0, 1);
        }
        for (int t : large) B.order.push_back(t);
        const int root_l = large.empty() ? -1 : B.build_sah(ns, ntri, 0);
        root = root_s < 0 ? root_l : root_l < 0 ? root_s : B.make_inner(root_l, root_s);
    } else if (!use_ref) {
        B.order.resize(ntri);
        for (int t = 0; t < ntri; ++t) B.order[t] = t;
        root = B.build_sah(0, ntri, 0);
    }

    // New node numbering: the first kTop nodes in breadth-first order, then depth-first preorder.
    const int n = (int)B.nodes.size();
    const int kTop = 2048;
    std::vector<int> newid(n, -1);
    int next = 0;
    {
        std::deque<int> q;
        q.push_back(root);
        while (!q.empty() && next < kTop) {
            int x = q.front();
            q.pop_front();
            newid[x] = next++;
            if (B.nodes[x].count == 0) { q.push_back(B.nodes[x].left); q.push_back(B.nodes[x].right); }
        }
        std::vector<int> st{root};
        while (!st.empty()) {
            int x = st.back();
            st.pop_back();
            if (newid[x] < 0) newid[x] = next++;
            if (B.nodes[x].count == 0) { st.push_back(B.nodes[x].right); st.push_back(B.nodes[x].left); }
        }
    }
    // Miss links: miss(left) = right, miss(right) = miss(parent), miss(root) = -1.
    std::vector<int> miss(n, -1);
    {
        std::vector<int> st{root};
        while (!st.empty()) {
            int x = st.back();
            st.pop_back();
            const BNode& N = B.nodes[x];
            if (N.count == 0) {
                miss[N.left] = newid[N.right];
                miss[N.right] = miss[x];
                st.push_back(N.right);
                st.push_back(N.left);
            }
        }
    }
    out->n_nodes = n;
    out->nodes.assign(2 * (size_t)n, make_float4(0, 0, 0, 0));
    out->n_tris = ntri;
    out->tris.assign(3 * (size_t)ntri, make_float4(0, 0, 0, 0));
    // nodes and triangles in their device layout, each host thread a range (every output slot is
    // written by exactly one thread)
    const unsigned nparts = host_parts(n);
    const size_t nper = ((size_t)n + nparts - 1) / nparts;
    parallel_parts(nparts, [&](unsigned part) {
        const int x1 = (int)std::min((size_t)n, (part + 1) * nper);
        for (int x = (int)std::min((size_t)n, part * nper); x < x1; ++x) {
            const BNode& N = B.nodes[x];
            float lo[3] = {N.lo[0], N.lo[1], N.lo[2]}, hi[3] = {N.hi[0], N.hi[1], N.hi[2]};
            pad_box(lo, hi);
            int child;
            if (N.count > 0) child = -1 - ((N.first << 3) | (N.count - 1));
            else child = newid[N.left];
            int i = newid[x];
            out->nodes[2 * (size_t)i + 0] = make_float4(lo[0], lo[1], lo[2], __builtin_bit_cast(float, child));
            out->nodes[2 * (size_t)i + 1] = make_float4(hi[0], hi[1], hi[2], __builtin_bit_cast(float, miss[x]));
        }
    });
    parallel_parts(parts, [&](unsigned part) {
        const int i1 = (int)std::min((size_t)ntri, (part + 1) * per);
        for (int i = (int)std::min((size_t)ntri, part * per); i < i1; ++i) {
            int t = B.order[i];
            const float* p = &B.v[9 * (size_t)t];
            out->tris[3 * (size_t)i + 0] = make_float4(p[0], p[1], p[2], __builtin_bit_cast(float, B.surf[t]));
            out->tris[3 * (size_t)i + 1] = make_float4(p[3], p[4], p[5], __builtin_bit_cast(float, t));
            float emin = INFINITY;
            for (int e = 0; e < 3; ++e) {
                const float* A = p + 3 * e;
                const float* Bv = p + 3 * ((e + 1) % 3);
                const float dx = Bv[0] - A[0], dy = Bv[1] - A[1], dz = Bv[2] - A[2];
                emin = std::min(emin, std::sqrt(dx * dx + dy * dy + dz * dz));
            }
            float band = emin > 0.0f ? kEdgeBandLength / emin : kEdgeBandMax;
            band = std::min(kEdgeBandMax, std::max(kEdgeBandMin, band));
            out->tris[3 * (size_t)i + 2] = make_float4(p[6], p[7], p[8], band);
        }
    });
    return true;
}

int occupied_z_slabs(const GeomImage& g, float* lo, float* hi) {
    std::vector<std::pair<float, float>> iv;
    iv.reserve(g.n_tris);
    for (int i = 0; i < g.n_tris; ++i) {
        const float4 a = g.tris[3 * (size_t)i], b = g.tris[3 * (size_t)i + 1], c = g.tris[3 * (size_t)i + 2];
        float zl = std::min(a.z, std::min(b.z, c.z)), zh = std::max(a.z, std::max(b.z, c.z));
        const float pad = 1e-5f * std::max(1.0f, std::max(std::fabs(zl), std::fabs(zh)));
        iv.push_back({zl - pad, zh + pad});
    }
    std::sort(iv.begin(), iv.end());
    std::vector<std::pair<float, float>> m;
    for (auto& v : iv) {
        if (!m.empty() && v.first <= m.back().second) m.back().second = std::max(m.back().second, v.second);
        else m.push_back(v);
    }
    // too many: close the narrowest gaps (a larger occupied set is still correct)
    while ((int)m.size() > kMaxZSlabs) {
        size_t best = 0;
        float gap = INFINITY;
        for (size_t i = 0; i + 1 < m.size(); ++i)
            if (m[i + 1].first - m[i].second < gap) { gap = m[i + 1].first - m[i].second; best = i; }
        m[best].second = std::max(m[best].second, m[best + 1].second);
        m.erase(m.begin() + best + 1);
    }
    for (size_t i = 0; i < m.size(); ++i) { lo[i] = m[i].first; hi[i] = m[i].second; }
    return (int)m.size();
}

void build_xy_grid(const GeomImage& g, GridImage* out, int tris_per_cell) {
    const double tpc = std::max(1, tris_per_cell);
    *out = GridImage();
    if (g.n_tris == 0) return;
    struct Box { float ax, bx, ay, by, zl, zh; };
    std::vector<Box> box(g.n_tris);
    for (int t = 0; t < g.n_tris; ++t) {
        Box& b = box[t];
        b.ax = b.ay = b.zl = INFINITY;
        b.bx = b.by = b.zh = -INFINITY;
        for (int c = 0; c < 3; ++c) {
            const float4 v = g.tris[3 * (size_t)t + c];
            b.ax = std::min(b.ax, v.x); b.bx = std::max(b.bx, v.x);
            b.ay = std::min(b.ay, v.y); b.by = std::max(b.by, v.y);
            b.zl = std::min(b.zl, v.z); b.zh = std::max(b.zh, v.z);
        }
    }
    // The grid covers the small triangles only: triangles spanning more than kBigTriangleCells cells
    // (the planes of a layer stack) are tested by every query from a short list instead. Their
    // extent must not set the grid's, so the bounds are refined a few times: grid over the current
    // set, mark the big triangles, bounds of the rest.
    std::vector<char> is_big(g.n_tris, 0);
    float xlo = 0, ylo = 0, xhi = 0, yhi = 0, padx = 0, pady = 0;
    int nx = 1, ny = 1;
    double wx = 1, wy = 1;
    for (int pass = 0; pass < 4; ++pass) {
        xlo = ylo = INFINITY;
        xhi = yhi = -INFINITY;
        int n_small = 0;
        for (int t = 0; t < g.n_tris; ++t) {
            if (is_big[t]) continue;
            ++n_small;
            xlo = std::min(xlo, box[t].ax); xhi = std::max(xhi, box[t].bx);
            ylo = std::min(ylo, box[t].ay); yhi = std::max(yhi, box[t].by);
        }
        if (n_small == 0) {  // every triangle is big: a one-cell grid with an empty cell
            xlo = ylo = 0.0f;
            xhi = yhi = 1.0f;
        }
        padx = 1e-5f * std::max(1.0f, std::max(std::fabs(xlo), std::fabs(xhi)));
        pady = 1e-5f * std::max(1.0f, std::max(std::fabs(ylo), std::fabs(yhi)));
        xlo -= padx; xhi += padx; ylo -= pady; yhi += pady;
        wx = std::max(1e-6f, xhi - xlo);
        wy = std::max(1e-6f, yhi - ylo);
        // about tris_per_cell triangles per cell (default 2), square-ish cells, at most 1024 x 1024
        const double cells = std::min(1048576.0, std::max(1.0, n_small / tpc));
        nx = (int)std::ceil(std::sqrt(cells * wx / wy));
        nx = std::max(1, std::min(1024, nx));
        ny = (int)std::ceil(cells / nx);
        ny = std::max(1, std::min(1024, ny));
        const double icx = nx / wx, icy = ny / wy;
        std::vector<char> next(g.n_tris, 0);
        int n_big = 0;
        for (int t = 0; t < g.n_tris; ++t) {
            // cells the triangle spans at this cell size (clamping ignored: a triangle outside the
            // current bounds counts in full)
            const double cx = std::floor((box[t].bx + padx - xlo) * icx) - std::floor((box[t].ax - padx - xlo) * icx) + 1;
            const double cy = std::floor((box[t].by + pady - ylo) * icy) - std::floor((box[t].ay - pady - ylo) * icy) + 1;
            if (is_big[t] || cx * cy > kBigTriangleCells) {
                next[t] = 1;
                ++n_big;
            }
        }
        if (n_big > kMaxBigTriangles) {
            // more large triangles than the list holds: no refinement, the grid covers every triangle
            std::fill(is_big.begin(), is_big.end(), 0);
            break;
        }
        if (next == is_big) break;
        is_big.swap(next);
    }
    // final bounds and size from the final marking
    {
        xlo = ylo = INFINITY;
        xhi = yhi = -INFINITY;
        int n_small = 0;
        for (int t = 0; t < g.n_tris; ++t) {
            if (is_big[t]) continue;
            ++n_small;
            xlo = std::min(xlo, box[t].ax); xhi = std::max(xhi, box[t].bx);
            ylo = std::min(ylo, box[t].ay); yhi = std::max(yhi, box[t].by);
        }
        if (n_small == 0) {
            xlo = ylo = 0.0f;
            xhi = yhi = 1.0f;
        }
        padx = 1e-5f * std::max(1.0f, std::max(std::fabs(xlo), std::fabs(xhi)));
        pady = 1e-5f * std::max(1.0f, std::max(std::fabs(ylo), std::fabs(yhi)));
        xlo -= padx; xhi += padx; ylo -= pady; yhi += pady;
        wx = std::max(1e-6f, xhi - xlo);
        wy = std::max(1e-6f, yhi - ylo);
        const double cells = std::min(1048576.0, std::max(1.0, n_small / tpc));
        nx = (int)std::ceil(std::sqrt(cells * wx / wy));
        nx = std::max(1, std::min(1024, nx));
        ny = (int)std::ceil(cells / nx);
        ny = std::max(1, std::min(1024, ny));
    }
    out->nx = nx;
    out->ny = ny;
    out->x0 = xlo;
    out->y0 = ylo;
    out->icx = (float)(nx / wx);
    out->icy = (float)(ny / wy);
    const size_t nc = (size_t)nx * ny;
    struct Span { int i0, i1, j0, j1; float zl, zh; };
    std::vector<Span> spans(g.n_tris);
    for (int t = 0; t < g.n_tris; ++t) {
        const Box& b = box[t];
        const float pz = 1e-5f * std::max(1.0f, std::max(std::fabs(b.zl), std::fabs(b.zh)));
        Span& sp = spans[t];
        sp.zl = b.zl - pz;
        sp.zh = b.zh + pz;
        sp.i0 = std::max(0, std::min(nx - 1, (int)std::floor((b.ax - padx - xlo) * out->icx)));
        sp.i1 = std::max(0, std::min(nx - 1, (int)std::floor((b.bx + padx - xlo) * out->icx)));
        sp.j0 = std::max(0, std::min(ny - 1, (int)std::floor((b.ay - pady - ylo) * out->icy)));
        sp.j1 = std::max(0, std::min(ny - 1, (int)std::floor((b.by + pady - ylo) * out->icy)));
    }
    auto as_float = [](int t) { float f; std::memcpy(&f, &t, sizeof(f)); return f; };
    // the big list: every triangle marked above (at most kMaxBigTriangles; they may lie outside the
    // grid's bounds), then, while there is room, triangles that span too many cells of the final grid
    for (int t = 0; t < g.n_tris; ++t) {
        if (!is_big[t]) continue;
        const Span& sp = spans[t];
        out->big.push_back(make_float4(sp.zl, sp.zh, as_float(t), 0.0f));
        for (int c = 0; c < 3; ++c) out->big.push_back(g.tris[3 * (size_t)t + c]);
    }
    for (int t = 0; t < g.n_tris && (int)(out->big.size() / 4) < kMaxBigTriangles; ++t) {
        if (is_big[t]) continue;
        const Span& sp = spans[t];
        const long long covered = (long long)(sp.i1 - sp.i0 + 1) * (sp.j1 - sp.j0 + 1);
        if (covered > kBigTriangleCells) {
            is_big[t] = 1;
            out->big.push_back(make_float4(sp.zl, sp.zh, as_float(t), 0.0f));
            for (int c = 0; c < 3; ++c) out->big.push_back(g.tris[3 * (size_t)t + c]);
        }
    }
    std::vector<unsigned int> count(nc, 0);
    for (int t = 0; t < g.n_tris; ++t) {
        if (is_big[t]) continue;
        const Span& sp = spans[t];
        for (int j = sp.j0; j <= sp.j1; ++j)
            for (int i = sp.i0; i <= sp.i1; ++i) count[(size_t)j * nx + i]++;
    }
    out->cells.resize(nc);
    unsigned int acc = 0;
    for (size_t c = 0; c < nc; ++c) {
        out->cells[c] = make_uint2(acc, count[c]);
        acc += count[c];
    }
    out->entries.resize(acc);
    std::vector<unsigned int> fill(nc);
    for (size_t c = 0; c < nc; ++c) fill[c] = out->cells[c].x;
    for (int t = 0; t < g.n_tris; ++t) {
        if (is_big[t]) continue;
        const Span& sp = spans[t];
        for (int j = sp.j0; j <= sp.j1; ++j)
            for (int i = sp.i0; i <= sp.i1; ++i)
                out->entries[fill[(size_t)j * nx + i]++] = make_float4(sp.zl, sp.zh, as_float(t), 0.0f);
    }
    // per cell: the z-intervals its triangles occupy, merged and reduced to at most 4 (a step whose
    // z-range misses them all cannot hit a triangle of the cell). The cell's entries are sorted by
    // z-low, so the entries of each interval are contiguous (every entry's z-range lies inside exactly
    // one interval and the intervals are disjoint and ordered); cell_runs keeps their counts.
    out->cell_z.assign(2 * nc, make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY));
    out->cell_runs.assign(nc, 0u);
    // cells are independent: up to 16 host threads, each a contiguous range of cells
    const unsigned parts = nc < 4096 ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t per = (nc + parts - 1) / parts;
    parallel_parts(parts, [&](unsigned part) {
        std::vector<std::pair<float, float>> iv, m;
        const size_t c_end = std::min(nc, (part + 1) * per);
        for (size_t c = part * per; c < c_end; ++c) {
            float4* ce = out->entries.data() + out->cells[c].x;
            const unsigned int cn = out->cells[c].y;
            std::sort(ce, ce + cn, [](const float4& a, const float4& b) {
                if (a.x != b.x) return a.x < b.x;
                int ta, tb;
                std::memcpy(&ta, &a.z, sizeof(ta));
                std::memcpy(&tb, &b.z, sizeof(tb));
                return ta < tb;
            });
            iv.clear();
            for (unsigned int k = 0; k < cn; ++k) iv.push_back({ce[k].x, ce[k].y});
            std::sort(iv.begin(), iv.end());
            m.clear();
            for (auto& v : iv) {
                if (!m.empty() && v.first <= m.back().second) m.back().second = std::max(m.back().second, v.second);
                else m.push_back(v);
            }
            while (m.size() > 4) {
                size_t best = 0;
                float gap = INFINITY;
                for (size_t q = 0; q + 1 < m.size(); ++q)
                    if (m[q + 1].first - m[q].second < gap) { gap = m[q + 1].first - m[q].second; best = q; }
                m[best].second = std::max(m[best].second, m[best + 1].second);
                m.erase(m.begin() + best + 1);
            }
            float z[8] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
            for (size_t q = 0; q < m.size(); ++q) { z[2 * q] = m[q].first; z[2 * q + 1] = m[q].second; }
            out->cell_z[2 * c] = make_float4(z[0], z[1], z[2], z[3]);
            out->cell_z[2 * c + 1] = make_float4(z[4], z[5], z[6], z[7]);
            unsigned int cnt[4] = {0, 0, 0, 0};
            bool split = true;
            for (unsigned int k = 0; k < cn; ++k) {
                size_t q = 0;
                while (q + 1 < m.size() && ce[k].x > m[q].second) ++q;
                if (!(ce[k].x >= m[q].first && ce[k].y <= m[q].second)) split = false;  // not inside one interval
                ++cnt[q];
            }
            for (int q = 0; q < 4; ++q) split = split && cnt[q] <= 255u;
            out->cell_runs[c] = split ? (cnt[0] | cnt[1] << 8 | cnt[2] << 16 | cnt[3] << 24) : 0xffffffffu;
        }
    });
}

// GenerateBVHTree replacement (mcml_intersection.cpp:316-344): a binned-SAH tree of this library
// returned in the reference's own BVHTree layout (FP64 boxes, leaves as (surfId, trIndex) runs,
// nodes listed children-before-parent with the root last, as the reference emits them), so callers
// of the reference API can prebuild input->bvhTree once and pass it to every launch.
BVHTree* generate_reference_tree(const Surface* surfaces, int numberOfSurfaces, std::string* err) {
    Builder B;
    int ntri = 0;
    for (int s = 0; s < numberOfSurfaces; ++s) ntri += std::max(0, surfaces[s].numberOfTriangles);
    B.v.resize(9 * (size_t)ntri);
    B.surf.resize(ntri);
    B.cen.resize(3 * (size_t)ntri);
    std::vector<std::pair<int, int>> ids(ntri);
    for (int s = 0, t = 0; s < numberOfSurfaces; ++s) {
        const Surface& S = surfaces[s];
        for (int j = 0; j < S.numberOfTriangles; ++j, ++t) {
            const xmc_ref_int3& T = S.triangles[j];
            const int id[3] = {T.x, T.y, T.z};
            for (int c = 0; c < 3; ++c) {
                if (id[c] < 0 || id[c] >= S.numberOfVertices) { *err = "vertex index out of range"; return nullptr; }
                for (int k = 0; k < 3; ++k) B.v[9 * (size_t)t + 3 * c + k] = (float)S.vertices[id[c]].cell[k];
            }
            for (int k = 0; k < 3; ++k)
                B.cen[3 * (size_t)t + k] = (B.v[9 * (size_t)t + k] + B.v[9 * (size_t)t + 3 + k] + B.v[9 * (size_t)t + 6 + k]) / 3.0f;
            B.surf[t] = s;
            ids[t] = {s, j};
        }
    }
    BVHTree* tree = new BVHTree;
    std::memset(tree, 0, sizeof(*tree));
    tree->numOfTriangles = ntri;
    tree->triangles = new Triangle[std::max(1, ntri)];
    if (ntri == 0) {
        tree->nodes = new BVHNode[1];
        std::memset(tree->nodes, 0, sizeof(BVHNode));
        tree->nodes[0].offset = 0;
        tree->nodes[0].numOfTriangles = 0;
        tree->nodes[0].leftNode = tree->nodes[0].rightNode = -1;
        tree->numOfNodes = 1;
        tree->root = 0;
        return tree;
    }
    B.order.resize(ntri);
    for (int t = 0; t < ntri; ++t) B.order[t] = t;
    const int root = B.build_sah(0, ntri, 0);
    for (int i = 0; i < ntri; ++i) {
        tree->triangles[i].surfId = ids[B.order[i]].first;
        tree->triangles[i].trIndex = ids[B.order[i]].second;
    }
    // exact FP64 boxes from the original vertices, children before parents (post-order)
    const int n = (int)B.nodes.size();
    tree->nodes = new BVHNode[n];
    tree->numOfNodes = n;
    std::vector<int> newid(n, -1);
    int next = 0;
    std::function<void(int)> emit = [&](int x) {
        const BNode& N = B.nodes[x];
        if (N.count == 0) { emit(N.left); emit(N.right); }
        BVHNode& o = tree->nodes[next];
        std::memset(&o, 0, sizeof(o));
        newid[x] = next++;
        if (N.count > 0) {
            double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int i = N.first; i < N.first + N.count; ++i) {
                const Surface& S = surfaces[tree->triangles[i].surfId];
                const xmc_ref_int3& T = S.triangles[tree->triangles[i].trIndex];
                for (int v : {T.x, T.y, T.z})
                    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], S.vertices[v].cell[k]); hi[k] = std::max(hi[k], S.vertices[v].cell[k]); }
            }
            for (int k = 0; k < 3; ++k) { o.Box.Ver1.cell[k] = lo[k]; o.Box.Ver2.cell[k] = hi[k]; }
            o.offset = N.first;
            o.numOfTriangles = N.count;
            o.leftNode = o.rightNode = -1;
        } else {
            const BVHNode& L = tree->nodes[newid[N.left]];
            const BVHNode& R = tree->nodes[newid[N.right]];
            for (int k = 0; k < 3; ++k) {
                o.Box.Ver1.cell[k] = std::min(L.Box.Ver1.cell[k], R.Box.Ver1.cell[k]);
                o.Box.Ver2.cell[k] = std::max(L.Box.Ver2.cell[k], R.Box.Ver2.cell[k]);
            }
            o.offset = -1;
            o.numOfTriangles = 0;
            o.leftNode = newid[N.left];
            o.rightNode = newid[N.right];
        }
    };
    emit(root);
    tree->root = newid[root];
    return tree;
}

}  // namespace xmc

extern "C" BVHTree* xmc_generate_bvh_tree(const Surface* surfaces, int numberOfSurfaces) {
    std::string err;
    if (!surfaces && numberOfSurfaces > 0) { xmc::set_error("surfaces is NULL"); return nullptr; }
    BVHTree* t = xmc::generate_reference_tree(surfaces, numberOfSurfaces, &err);
    if (!t) xmc::set_error(err);
    return t;
}

extern "C" void xmc_free_bvh_tree(BVHTree* tree) {
    if (!tree) return;
    delete[] tree->nodes;
    delete[] tree->triangles;
    delete tree;
}
