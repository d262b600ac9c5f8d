// Compiled plane passes of the two-sweep 3D step, one per (x plan, y plan,
// CTAs per plane) of the registry: the whole padded x-y plane in one CTA, or
// spread over a cluster of 2 or 4 CTAs (rows and columns split among them).
// Arguments: <type, nx, x E, x radices, ny, y E, y radices, threads, CTAs per plane>.
// Built where a single-handle n^3 step measured faster than the four axis passes
// on B200, or within a few percent of the best plane form (left to the autotuner).
// Not built, slower than four axis passes (us per n^3 step, four passes first):
// complex128 96^2 on 1 / 2 / 4 CTAs (30.1 vs 35.0 / 40.2 / 40.3), 128^2 on 4
// (57.8 vs 71.3); complex64 128^2 on 2 / 4 (47.1 vs 43.3 / 55.3, one CTA 36.4),
// 160^2 on 4 (92.1 vs 112.8), 256^2 on 8 (169 KB per CTA: 310 vs 470 us, C2's grid; the
// same bits as the four passes).
#include "ses_plane.cuh"

namespace sesk {
void register_planes(std::vector<PlaneEntry<float>>& f, std::vector<PlaneEntry<double>>& d) {
    f.push_back(make_plane_entry<float, 32, 8, 8, 4, 1, 32, 8, 8, 4, 1, 128>());
    f.push_back(make_plane_entry<float, 32, 8, 8, 4, 1, 32, 8, 8, 4, 1, 64, 2>());
    f.push_back(make_plane_entry<float, 48, 12, 12, 4, 1, 48, 12, 12, 4, 1, 192>());
    f.push_back(make_plane_entry<float, 48, 12, 12, 4, 1, 48, 12, 12, 4, 1, 96, 2>());
    f.push_back(make_plane_entry<float, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 512>());
    f.push_back(make_plane_entry<float, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 256, 2>());
    f.push_back(make_plane_entry<float, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 128, 4>());
    f.push_back(make_plane_entry<float, 96, 12, 6, 4, 4, 96, 24, 12, 8, 1, 384>());
    f.push_back(make_plane_entry<float, 96, 12, 6, 4, 4, 96, 24, 12, 8, 1, 192, 2>());
    f.push_back(make_plane_entry<float, 96, 12, 6, 4, 4, 96, 24, 12, 8, 1, 96, 4>());
    f.push_back(make_plane_entry<float, 128, 16, 16, 8, 1, 128, 16, 16, 8, 1, 512>());
    d.push_back(make_plane_entry<double, 32, 8, 8, 4, 1, 32, 8, 8, 4, 1, 128>());
    d.push_back(make_plane_entry<double, 32, 8, 8, 4, 1, 32, 8, 8, 4, 1, 64, 2>());
    d.push_back(make_plane_entry<double, 48, 12, 4, 4, 3, 48, 12, 4, 4, 3, 192>());
    d.push_back(make_plane_entry<double, 48, 12, 4, 4, 3, 48, 12, 4, 4, 3, 96, 2>());
    d.push_back(make_plane_entry<double, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 512>());
    d.push_back(make_plane_entry<double, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 256, 2>());
    d.push_back(make_plane_entry<double, 64, 8, 8, 8, 1, 64, 8, 8, 8, 1, 128, 4>());
}
}  // namespace sesk
