/*
 * projection_oracle.c -- CPU restatement of the two steps either side of the
 * pressure solve in a FLIP projection, for the GPU parity tests.  TEST
 * INFRASTRUCTURE ONLY: the product never links or calls this file.
 *
 *  - fraction_inside(bl, br, tl, tr): SIMD_UAAMG/levelset_util.cpp:23-100
 *    (and the two-sample form, :4-13)
 *  - FLIP_Solver_OpenVDB::calculate_face_weights: FLIP_vdb/FLIP_vdb.cpp:2669-2752
 *  - FLIP_Solver_OpenVDB::apply_pressure_gradient: FLIP_vdb/FLIP_vdb.cpp:2571-2667
 *  - vdb_velocity_extrapolator::union_extrapolate, the layers after its
 *    topology steps: FLIP_vdb/vdb_velocity_extrapolator.cpp:611-659
 *  - FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids, its value passes:
 *    FLIP_vdb/FLIP_vdb.cpp:2856-2938
 *
 * Compiled with -ffp-contract=off: every float operation is the reference's,
 * in its order, unfused.  Grids are flattened leaf grids (OpenVDB leaf
 * layout, ConstAccessor::getValue semantics through oracle_common.h).
 */
#include "uaamg_oracle.h"

#include "oracle_common.h"

/* levelset_util.cpp:4-13 */
static float fi2(float phi_left, float phi_right) {
    if (phi_left < 0 && phi_right < 0) return 1;
    if (phi_left < 0 && phi_right >= 0) return phi_left / (phi_left - phi_right);
    if (phi_left >= 0 && phi_right < 0) return phi_right / (phi_right - phi_left);
    return 0;
}

/* levelset_util.cpp:15-20 */
static void cycle(float* arr, int size) {
    float t = arr[0];
    for (int i = 0; i < size - 1; ++i) arr[i] = arr[i + 1];
    arr[size - 1] = t;
}

/* levelset_util.cpp:23-100 */
float orc_fraction_inside4(float phi_bl, float phi_br, float phi_tl, float phi_tr) {
    int inside_count = (phi_bl < 0 ? 1 : 0) + (phi_tl < 0 ? 1 : 0) + (phi_br < 0 ? 1 : 0) + (phi_tr < 0 ? 1 : 0);
    float list[4] = {phi_bl, phi_br, phi_tr, phi_tl};
    if (inside_count == 4) return 1;
    if (inside_count == 3) {
        while (list[0] < 0) cycle(list, 4);
        float side0 = 1 - fi2(list[0], list[3]);
        float side1 = 1 - fi2(list[0], list[1]);
        return 1 - 0.5f * side0 * side1;
    }
    if (inside_count == 2) {
        int guard = 0;
        while ((list[0] >= 0 || !(list[1] < 0 || list[2] < 0)) && guard++ < 4) cycle(list, 4);
        if (list[1] < 0) {
            float side_left = fi2(list[0], list[3]);
            float side_right = fi2(list[1], list[2]);
            return 0.5f * (side_left + side_right);
        }
        float middle_point = 0.25f * (list[0] + list[1] + list[2] + list[3]);
        if (middle_point < 0) {
            float area = 0;
            float side1 = 1 - fi2(list[0], list[3]);
            float side3 = 1 - fi2(list[2], list[3]);
            area += 0.5f * side1 * side3;
            float side2 = 1 - fi2(list[2], list[1]);
            float side0 = 1 - fi2(list[0], list[1]);
            area += 0.5f * side0 * side2;
            return 1 - area;
        }
        float area = 0;
        float side0 = fi2(list[0], list[1]);
        float side1 = fi2(list[0], list[3]);
        area += 0.5f * side0 * side1;
        float side2 = fi2(list[2], list[1]);
        float side3 = fi2(list[2], list[3]);
        area += 0.5f * side2 * side3;
        return area;
    }
    if (inside_count == 1) {
        while (list[0] >= 0) cycle(list, 4);
        float side0 = fi2(list[0], list[3]);
        float side1 = fi2(list[0], list[1]);
        return 0.5f * side0 * side1;
    }
    return 0;
}

/* std::max(0.f, std::min(v, 1.f)) */
static float clamp01(float v) {
    float m = (1.f < v) ? 1.f : v;
    return (0.f < m) ? m : 0.f;
}

/* FLIP_vdb.cpp:2680-2745: the weights of the active voxels of the given
 * topology (masks NULL: all), (1, 1, 1) at the others. */
void orc_face_weights(int64_t solid_n, const int32_t* solid_origins, const float* solid_values, float solid_bg,
                      int64_t n, const int32_t* origins, const uint64_t* masks, float* out) {
    ogrid solid;
    const float bg[3] = {solid_bg, 0.f, 0.f};
    ogrid_init(&solid, solid_n, solid_origins, NULL, solid_values, 1, bg);
#pragma omp parallel for schedule(static)
    for (int64_t li = 0; li < n; ++li) {
        for (int off = 0; off < LSZ; ++off) {
            float* o = out + ((size_t)li * LSZ + off) * 3;
            if (masks && !mbit(masks + 8 * li, off)) {
                o[0] = o[1] = o[2] = 1.f;
                continue;
            }
            const int gx = origins[3 * li] + (off >> 6), gy = origins[3 * li + 1] + ((off >> 3) & 7),
                      gz = origins[3 * li + 2] + (off & 7);
            float ssdf[2][2][2];
            for (int ii = 0; ii < 2; ii++)
                for (int jj = 0; jj < 2; jj++)
                    for (int kk = 0; kk < 2; kk++) ssdf[ii][jj][kk] = ogrid_get(&solid, gx + ii, gy + jj, gz + kk, 0);
            float w[3];
            w[0] = clamp01(1.0f - orc_fraction_inside4(ssdf[0][0][0], ssdf[0][1][0], ssdf[0][0][1], ssdf[0][1][1]));
            w[1] = clamp01(1.0f - orc_fraction_inside4(ssdf[0][0][0], ssdf[0][0][1], ssdf[1][0][0], ssdf[1][0][1]));
            w[2] = clamp01(1.0f - orc_fraction_inside4(ssdf[0][0][0], ssdf[1][0][0], ssdf[0][1][0], ssdf[1][1][0]));
            for (int c = 0; c < 3; c++)
                if (w[c] < 1e-2f) w[c] = 0.f;
            o[0] = w[0];
            o[1] = w[1];
            o[2] = w[2];
        }
    }
    leafmap_free(&solid.map);
}

/* FLIP_vdb.cpp:2584-2663 for one channel.  The pressure grid is given by its
 * leaves, DOF masks (isValueOn) and values (getValue; 0 outside the leaves).
 * Outputs as the GPU entry point: velocity, new active masks, update and
 * reflected values (the input value where there is no update). */
void orc_pressure_gradient(int64_t phi_n, const int32_t* phi_origins, const float* phi_values, float phi_bg,
                           int64_t fw_n, const int32_t* fw_origins, const float* fw_values, const float* fw_bg3,
                           int64_t sv_n, const int32_t* sv_origins, const float* sv_values, const float* sv_bg3,
                           int64_t p_n, const int32_t* p_origins, const uint64_t* p_masks, const float* p_values,
                           float in_dt, float dx, float friction, int channel,
                           int64_t v_n, const int32_t* v_origins, const uint64_t* v_masks, const float* v_values,
                           float* v_out, uint64_t* mask_out, float* update_out, float* reflected_out) {
    ogrid phi, fw, sv, pg;
    const float pbg[3] = {phi_bg, 0.f, 0.f}, zero[3] = {0.f, 0.f, 0.f};
    ogrid_init(&phi, phi_n, phi_origins, NULL, phi_values, 1, pbg);
    ogrid_init(&fw, fw_n, fw_origins, NULL, fw_values, 3, fw_bg3);
    ogrid_init(&sv, sv_n, sv_origins, NULL, sv_values, 3, sv_bg3);
    ogrid_init(&pg, p_n, p_origins, p_masks, p_values, 1, zero);
#pragma omp parallel for schedule(static)
    for (int64_t li = 0; li < v_n; ++li) {
        uint64_t m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int off = 0; off < LSZ; ++off) {
            const size_t i = (size_t)li * LSZ + off;
            float updated_vel = v_values[i];
            float reflected_vel = updated_vel;
            float vel_update = 0.0f;
            int has_update = 0;
            v_out[i] = v_values[i];
            if (v_masks && !mbit(v_masks + 8 * li, off)) {
                if (update_out) update_out[i] = v_values[i];
                if (reflected_out) reflected_out[i] = v_values[i];
                continue;
            }
            int g[3] = {v_origins[3 * li] + (off >> 6), v_origins[3 * li + 1] + ((off >> 3) & 7),
                        v_origins[3 * li + 2] + (off & 7)};
            int lo[3] = {g[0], g[1], g[2]};
            lo[channel] -= 1;
            float face_weight = ogrid_get(&fw, g[0], g[1], g[2], channel);
            if (face_weight > 0.0f) {
                int32_t a = leafmap_find(&pg.map, g[0], g[1], g[2]);
                int32_t b = leafmap_find(&pg.map, lo[0], lo[1], lo[2]);
                int has_pressure = a >= 0 && mbit(p_masks + 8 * a, voff(g[0], g[1], g[2]));
                int has_pressure_below = b >= 0 && mbit(p_masks + 8 * b, voff(lo[0], lo[1], lo[2]));
                if (has_pressure || has_pressure_below) has_update = 1;
                if (has_update) {
                    float phi_this = ogrid_get(&phi, g[0], g[1], g[2], 0);
                    float phi_below = ogrid_get(&phi, lo[0], lo[1], lo[2], 0);
                    float p_this = ogrid_get(&pg, g[0], g[1], g[2], 0);
                    float p_below = ogrid_get(&pg, lo[0], lo[1], lo[2], 0);
                    float theta = 1.0f;
                    if (phi_this >= 0 || phi_below >= 0) {
                        theta = fi2(phi_below, phi_this);
                        if (theta < 0.02f) theta = 0.02f;
                    }
                    vel_update = -in_dt * (float)(p_this - p_below) / dx / theta;
                    updated_vel += vel_update;
                    reflected_vel = updated_vel + vel_update;
                    if (face_weight < 1.0f) {
                        float solid_vel = ogrid_get(&sv, g[0], g[1], g[2], channel);
                        float solid_fraction = (1.0f - face_weight) * friction;
                        updated_vel = (1.0f - solid_fraction) * updated_vel + (solid_fraction)*solid_vel;
                    }
                }
            }
            if (has_update) {
                v_out[i] = updated_vel;
                m[off >> 6] |= 1ull << (off & 63);
                if (update_out) update_out[i] = vel_update;
                if (reflected_out) reflected_out[i] = reflected_vel;
            } else {
                if (update_out) update_out[i] = v_values[i];
                if (reflected_out) reflected_out[i] = v_values[i];
            }
        }
        for (int w = 0; w < 8; ++w) mask_out[8 * li + w] = m[w];
    }
    leafmap_free(&phi.map);
    leafmap_free(&fw.map);
    leafmap_free(&sv.map);
    leafmap_free(&pg.map);
}

/* vdb_velocity_extrapolator.cpp:611-659 for one channel on flattened grids:
 * the output grid (n_out leaves, values and active masks updated in place)
 * and the fill set (fill_leaf[e]: output leaf, fill_masks[e]: voxels still to
 * fill).  Each layer snapshots the channel's topology (valid_vel_topo) and
 * fills every fill voxel with an active face neighbour by the mean of those
 * neighbours, -x, +x, -y, +y, -z, +z. */
void orc_extrapolate_channel(int n_layer, int64_t n_out, const int32_t* out_origins, float* values,
                             uint64_t* masks, int64_t n_fill, const int32_t* fill_leaf, const uint64_t* fill_masks) {
    if (n_out <= 0 || n_fill <= 0) return;
    leafmap map;
    leafmap_init(&map, n_out, out_origins);
    uint64_t* snap = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n_out * 8);
    uint64_t* rem = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n_fill * 8);
    memcpy(rem, fill_masks, sizeof(uint64_t) * (size_t)n_fill * 8);
    for (int ilayer = 0; ilayer < n_layer; ilayer++) {
        memcpy(snap, masks, sizeof(uint64_t) * (size_t)n_out * 8);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < n_fill; ++e) {
            const int32_t li = fill_leaf[e];
            const int32_t* o = out_origins + 3 * li;
            for (int off = 0; off < LSZ; ++off) {
                if (!mbit(rem + 8 * e, off)) continue;
                int temp_weight = 0;
                float temp_weighted_sum_val = 0;
                for (int d = 0; d < 6; d++) {
                    int direction = d / 2;
                    int positive = d % 2;
                    int neib[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
                    if (positive) neib[direction]++;
                    else neib[direction]--;
                    int32_t nl = leafmap_find(&map, neib[0], neib[1], neib[2]);
                    if (nl >= 0 && mbit(snap + 8 * nl, voff(neib[0], neib[1], neib[2]))) {
                        temp_weight++;
                        temp_weighted_sum_val += values[(size_t)nl * LSZ + voff(neib[0], neib[1], neib[2])];
                    }
                }
                if (temp_weight != 0) {
                    values[(size_t)li * LSZ + off] = temp_weighted_sum_val / temp_weight;
                    masks[8 * li + (off >> 6)] |= 1ull << (off & 63);
                    rem[8 * e + (off >> 6)] &= ~(1ull << (off & 63));
                }
            }
        }
    }
    free(snap);
    free(rem);
    leafmap_free(&map);
}

/* FLIP_Solver_OpenVDB::immerse_liquid_phi_in_solids, the value passes
 * (FLIP_vdb.cpp:2856-2938) over the liquid SDF's leaves as they were before
 * the 26-neighbour dilation (the reference's LeafManager is built at :2876,
 * before the dilation at :2881, and reused at :2938).  A leaf is processed
 * when the solid SDF has a leaf at its origin (probeConstLeaf).
 *   pass 1 (:2860-2877): active voxels whose solid SDF sampled at the voxel
 *     centre is negative get phi - 0.5 dx; the result is the reference copy;
 *   pass 2 (:2883-2938): voxels active after the dilation (the voxel or one
 *     of its 26 neighbours active) with a negative solid sample take the least
 *     of 3 dx and the reference values of the face neighbours visited in the
 *     order +x, -x, +y, -y, +z, -z up to the first negative one, if there is
 *     one; else a negative value becomes max(background, -solid).
 * values_out [n][512]: the liquid values after both passes. */
void orc_immerse_liquid_phi(int64_t solid_n, const int32_t* solid_origins, const float* solid_values, float solid_bg,
                            int64_t n, const int32_t* origins, const uint64_t* masks, const float* values,
                            float liquid_bg, float dx, float* values_out) {
    ogrid solid;
    const float sbg[3] = {solid_bg, 0.f, 0.f};
    ogrid_init(&solid, solid_n, solid_origins, NULL, solid_values, 1, sbg);
    float* ref = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1) * LSZ);
    memcpy(ref, values, sizeof(float) * (size_t)n * LSZ);
    const float half_dx = 0.5f * dx, three_dx = dx * 3.0f;
#pragma omp parallel for schedule(static)
    for (int64_t li = 0; li < n; ++li) {
        const int32_t* o = origins + 3 * li;
        if (leafmap_find(&solid.map, o[0], o[1], o[2]) < 0) continue;
        for (int off = 0; off < LSZ; ++off) {
            if (masks && !mbit(masks + 8 * li, off)) continue;
            float s = box_sample(&solid, o[0] + (off >> 6) + 0.5, o[1] + ((off >> 3) & 7) + 0.5, o[2] + (off & 7) + 0.5);
            if (s < 0) ref[li * LSZ + off] = values[li * LSZ + off] - half_dx;
        }
    }
    ogrid refg;
    const float lbg[3] = {liquid_bg, 0.f, 0.f};
    ogrid_init(&refg, n, origins, masks, ref, 1, lbg);
    memcpy(values_out, ref, sizeof(float) * (size_t)n * LSZ);
#pragma omp parallel for schedule(static)
    for (int64_t li = 0; li < n; ++li) {
        const int32_t* o = origins + 3 * li;
        if (leafmap_find(&solid.map, o[0], o[1], o[2]) < 0) continue;
        for (int off = 0; off < LSZ; ++off) {
            const int g[3] = {o[0] + (off >> 6), o[1] + ((off >> 3) & 7), o[2] + (off & 7)};
            int on = 0; /* active after one NN_FACE_EDGE_VERTEX dilation */
            for (int a = -1; a <= 1 && !on; ++a)
                for (int b = -1; b <= 1 && !on; ++b)
                    for (int c = -1; c <= 1 && !on; ++c) {
                        const int x = g[0] + a, y = g[1] + b, z = g[2] + c;
                        const int32_t nl = leafmap_find(&refg.map, x, y, z);
                        if (nl >= 0 && (!masks || mbit(masks + 8 * nl, voff(x, y, z)))) on = 1;
                    }
            if (!on) continue;
            float s = box_sample(&solid, g[0] + 0.5, g[1] + 0.5, g[2] + 0.5);
            if (!(s < 0)) continue;
            int found = 0;
            float min_fluid = three_dx;
            for (int i = 0; i < 6 && !found; i++) {
                int comp = i / 2, positive = (i % 2 == 0);
                int t[3] = {g[0], g[1], g[2]};
                t[comp] += positive ? 1 : -1;
                float r = ogrid_get(&refg, t[0], t[1], t[2], 0);
                min_fluid = (r < min_fluid) ? r : min_fluid; /* std::min */
                found |= (r < 0);
            }
            float* v = values_out + li * LSZ + off;
            if (found) {
                *v = min_fluid;
            } else if (*v < 0) {
                float ns = -s;
                *v = (liquid_bg < ns) ? ns : liquid_bg; /* std::max(background, -solid) */
            }
        }
    }
    leafmap_free(&refg.map);
    leafmap_free(&solid.map);
    free(ref);
}
