// Soundness of the 3D node bound (gquery_b200/csrc/sil_filter.h) on a real scene: the
// SNCH pair records and silhouette records a host build produced (raw 32-bit words of
// gq_spair3_t and gq_sile_t, as gq_scene_ref_array exports them) and a set of query
// points.  For every query the checker walks the whole tree; wherever the bound in its
// delta or cone form excludes a child whose parent it admitted, it runs the kernels'
// FP32 silhouette test on every record below that child (boundary records always
// count as silhouettes).  Excluded subtrees are disjoint, so a query costs at most one
// test per record.  Prints one JSON line of counts; a non-zero "unsound" is a failure.
//
// Usage: sil_node_check pairs.bin sils.bin queries.bin coord_bound
// Build: g++ -O2 -ffp-contract=off -I gquery_b200/csrc tests/sil_node_check.cpp
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "layout.h"
#include "sil_filter.h"
#include "sil_ref.h"

namespace {

template <class T>
std::vector<T> read_all(const char *path) {
    std::vector<T> v;
    FILE *f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / sizeof(T));
    if (!v.empty() && std::fread(v.data(), sizeof(T), v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

struct Scene {
    std::vector<gq_spair3_t> pairs;
    std::vector<gq_sile_t> sils;
};

// Whether any record below child reference `ref` is a silhouette for x.
bool subtree_has_silhouette(const Scene &s, int ref, V x, long long &tested) {
    if (ref < 0) {
        if (ref == INT32_MIN) return false;  // leaf without silhouettes
        for (size_t j = (size_t)~ref; j < s.sils.size(); ++j) {
            const gq_sile_t &r = s.sils[j];
            ++tested;
            const bool boundary = (r.flags & GQ_ITEM_VALID) != 0;
            if (boundary || reference_silhouette(V{r.ax, r.ay, r.az}, V{r.bx, r.by, r.bz}, V{r.n0x, r.n0y, r.n0z},
                                                 V{r.n1x, r.n1y, r.n1z}, x))
                return true;
            if (r.flags & GQ_ITEM_LAST) break;
        }
        return false;
    }
    const gq_spair3_t &p = s.pairs[(size_t)ref];
    return subtree_has_silhouette(s, p.ref_l, x, tested) || subtree_has_silhouette(s, p.ref_r, x, tested);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s pairs.bin sils.bin queries.bin coord_bound\n", argv[0]);
        return 2;
    }
    Scene s;
    s.pairs = read_all<gq_spair3_t>(argv[1]);
    s.sils = read_all<gq_sile_t>(argv[2]);
    const std::vector<V> q = read_all<V>(argv[3]);
    const float bound = (float)std::atof(argv[4]);
    if (s.pairs.empty() || s.sils.empty() || q.empty()) {
        std::fprintf(stderr, "empty input\n");
        return 2;
    }
    long long children = 0, ex_delta = 0, ex_cone = 0, ex_any = 0, unsound = 0, tested = 0;
    std::vector<int> stack;
    for (const V &x : q) {
        const float m = sil_node_margin(std::fmax(std::fabs(x.x), std::fmax(std::fabs(x.y), std::fabs(x.z))), bound);
        stack.assign(1, 0);  // pair 0: the root's children
        while (!stack.empty()) {
            const gq_spair3_t &p = s.pairs[(size_t)stack.back()];
            stack.pop_back();
            for (int c = 0; c < 2; ++c) {
                const float lo[3] = {c ? p.r_lox : p.l_lox, c ? p.r_loy : p.l_loy, c ? p.r_loz : p.l_loz};
                const float hi[3] = {c ? p.r_hix : p.l_hix, c ? p.r_hiy : p.l_hiy, c ? p.r_hiz : p.l_hiz};
                const float *b = c ? p.r_b : p.l_b;
                const int ref = c ? p.ref_r : p.ref_l;
                const float cx = sil_node_centre(lo[0], hi[0]), cy = sil_node_centre(lo[1], hi[1]),
                            cz = sil_node_centre(lo[2], hi[2]);
                const bool ed = sil_node_excluded_delta(cx, cy, cz, b, x.x, x.y, x.z, m);
                const bool ec = sil_node_excluded_cone(cx, cy, cz, b, x.x, x.y, x.z, m);
                ++children;
                ex_delta += ed;
                ex_cone += ec;
                if (ed || ec) {
                    ++ex_any;
                    if (subtree_has_silhouette(s, ref, x, tested)) {
                        if (unsound < 3)
                            std::fprintf(stderr, "unsound: child %d of pair excluded at x=(%a %a %a)\n", ref, x.x, x.y,
                                         x.z);
                        ++unsound;
                    }
                } else if (ref >= 0) {
                    stack.push_back(ref);
                }
            }
        }
    }
    std::printf("{\"queries\": %zu, \"children\": %lld, \"excluded\": %lld, \"delta\": %lld, \"cone\": %lld, "
                "\"records_tested\": %lld, \"unsound\": %lld}\n",
                q.size(), children, ex_any, ex_delta, ex_cone, tested, unsound);
    return unsound ? 1 : 0;
}
