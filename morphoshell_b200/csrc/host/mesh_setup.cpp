// One-off mesh set-up: topology, patch fitting, derivative coefficients,
// lumped masses and the characteristic scales that fix dt, damping and the
// dialling schedule.  Each function follows the reference file named above
// it; the formulas are kept term for term so that the scalars (and hence dt
// and the step counts) come out the same.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <exception>
#include <iterator>
#include <random>
#include <thread>
#include <vector>

#include "host.hpp"
#include "patch_fit.hpp"
#include "small_linalg.hpp"

namespace msb {

namespace {

inline double norm3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }

double vmin(const std::vector<double>& v, size_t* arg = nullptr) {
    auto it = std::min_element(v.begin(), v.end());
    if (arg) *arg = static_cast<size_t>(std::distance(v.begin(), it));
    return *it;
}
double vmax(const std::vector<double>& v, size_t* arg = nullptr) {
    auto it = std::max_element(v.begin(), v.end());
    if (arg) *arg = static_cast<size_t>(std::distance(v.begin(), it));
    return *it;
}

}  // namespace

// source_files/kahan_sum.cpp:32-49
double kahan_sum(const std::vector<double>& vec) {
    double sum = 0.0, comp = 0.0;
    for (double x : vec) {
        volatile double y = x - comp;
        volatile double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    return sum;
}

// calc_triangles_incident_on_nodes.cpp:47-53, calc_node_neighbours.cpp,
// calc_triangle_adjacencies.cpp, calc_edges.cpp and calc_mesh_info.cpp:50-185.
void calc_mesh_info(std::vector<Node>& nodes, const DMat& P, std::vector<Tri>& triangles, std::vector<Edge>& edges,
                    Stuff& stuff, Log& log) {
    // Incident triangles, in triangle order.
    for (auto& node : nodes) node.incident_tri_ids.clear();
    for (const auto& tri : triangles)
        for (int v : tri.vertex_ids) nodes.at(v).incident_tri_ids.push_back(tri.id);
    // 1-rings, sorted and unique (nodes independent: in parallel ranges).
    const int nthreads = setup_threads(std::max((int)nodes.size(), (int)triangles.size()));
    parallel_ranges((int)nodes.size(), nthreads, [&](int n0, int n1, int) {
        for (int n = n0; n < n1; ++n) {
            Node& node = nodes[n];
            node.neighbour_node_ids.clear();
            for (int t : node.incident_tri_ids)
                for (int v : triangles[t].vertex_ids)
                    if (v != node.id) node.neighbour_node_ids.push_back(v);
            std::sort(node.neighbour_node_ids.begin(), node.neighbour_node_ids.end());
            node.neighbour_node_ids.erase(
                std::unique(node.neighbour_node_ids.begin(), node.neighbour_node_ids.end()),
                node.neighbour_node_ids.end());
        }
    });
    // Edge-sharing triangles (triangles independent).
    parallel_ranges((int)triangles.size(), nthreads, [&](int t0, int t1, int) {
        std::vector<int> cand;
        for (int ti = t0; ti < t1; ++ti) {
            Tri& tri = triangles[ti];
            cand.clear();
            for (int v : tri.vertex_ids)
                for (int t : nodes[v].incident_tri_ids)
                    if (t != tri.id) cand.push_back(t);
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            tri.edge_sharing_tri_ids.clear();
            for (int t : cand) {
                int common = 0;
                for (int a : tri.vertex_ids)
                    for (int b : triangles[t].vertex_ids) common += (a == b);
                if (common == 2) tri.edge_sharing_tri_ids.push_back(t);
            }
        }
    });
    for (const auto& tri : triangles)
        if (tri.edge_sharing_tri_ids.size() < 1 || tri.edge_sharing_tri_ids.size() > 3)
            throw std::runtime_error(
                "Error: Problem with triangle (edge-sharing) adjacencies or edges setup. "
                "Either there is a bug, or some mesh pathology; investigate further!");
    // Edges (i, j), i < j, in lexicographic order.
    edges.clear();
    edges.reserve(3 * static_cast<size_t>(stuff.num_tris));
    for (const auto& node : nodes)
        for (int nb : node.neighbour_node_ids)
            if (nb > node.id) {
                Edge e;
                e.node_ids = {node.id, nb};
                if (edges.size() >= static_cast<size_t>(INT_MAX))
                    throw std::overflow_error("edge count overflowed int");
                e.id = static_cast<int>(edges.size());
                edges.push_back(e);
            }
    stuff.num_edges = static_cast<int>(edges.size());
    // Each edge's triangles: the common incident triangles of its ends (the
    // incidence lists are in triangle order, so already sorted; edges
    // independent).
    parallel_ranges((int)edges.size(), nthreads, [&](int e0, int e1, int) {
        std::vector<int> common;
        for (int ei = e0; ei < e1; ++ei) {
            Edge& e = edges[ei];
            const std::vector<int>& a = nodes[e.node_ids[0]].incident_tri_ids;
            const std::vector<int>& b = nodes[e.node_ids[1]].incident_tri_ids;
            common.clear();
            std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(common));
            if (common.size() == 1) {
                e.is_boundary = true;
                e.adjacent_tri_ids = common;
            } else if (common.size() == 2) {
                e.is_boundary = false;
                e.adjacent_tri_ids = common;
            } else {
                throw std::runtime_error(
                    "Something has gone very wrong in calc_edges, because the nodes at each end of an edge "
                    "should have either one or two incident triangles in common, but the code thinks it's "
                    "found an exception. Investigate!");
            }
        }
    });
    std::vector<int> cursor(stuff.num_tris, 0);
    for (const auto& e : edges)
        for (int t : e.adjacent_tri_ids) {
            if (cursor[t] < 3) triangles[t].edge_ids[cursor[t]] = e.id;
            cursor[t] += 1;
        }

    stuff.num_dofs = 3 * stuff.num_nodes;
    stuff.num_continuum_quantities = 15 * stuff.num_tris;
    stuff.num_boundary_edges = 0;
    std::vector<double> bedge_len;
    for (const auto& e : edges)
        if (e.is_boundary) {
            stuff.num_boundary_edges += 1;
            nodes[e.node_ids[0]].is_boundary = true;
            nodes[e.node_ids[1]].is_boundary = true;
            int i = e.node_ids[0], j = e.node_ids[1];
            bedge_len.push_back(norm3(P(i, 0) - P(j, 0), P(i, 1) - P(j, 1), P(i, 2) - P(j, 2)));
        }
    stuff.num_boundary_nodes = 0;
    for (const auto& node : nodes) stuff.num_boundary_nodes += node.is_boundary ? 1 : 0;
    for (auto& tri : triangles) {
        tri.is_boundary = false;
        for (int v : tri.vertex_ids) tri.is_boundary = tri.is_boundary || nodes[v].is_boundary;
    }
    double perimeter = kahan_sum(bedge_len);
    stuff.sample_char_length = perimeter;
    log << "Reference perimeter = " << perimeter << std::endl;
    log << "Number of edges = " << stuff.num_edges << std::endl;
    log << "Number of boundary edges = " << stuff.num_boundary_edges << std::endl;
    log << "Number of non-boundary edges = " << stuff.num_edges - stuff.num_boundary_edges << std::endl;
    log << "Number of holes in mesh = " << 1 + stuff.num_edges - stuff.num_nodes - stuff.num_tris << std::endl;
    log << "Number of boundary nodes = " << stuff.num_boundary_nodes << std::endl;
    if (3 * stuff.num_tris != 2 * stuff.num_edges - stuff.num_boundary_edges)
        throw std::runtime_error(
            "Something has gone wrong in calculating triangle adjacencies and/or "
            "edges: the current edge and triangle counts violate a topological identity.");
    if (1 + stuff.num_edges - stuff.num_nodes - stuff.num_tris < 0)
        throw std::runtime_error(
            "Something is very wrong with the mesh, because the code thinks it has a "
            "negative number of holes! A first thing to check is that all nodes touch at least one tri.");

    // Areas (Tri_Class.cpp:31-36), smallest altitudes, aspect ratios and
    // centroids per triangle (triangles independent); the sum and the minima
    // run over them in triangle order afterwards.
    const int T = static_cast<int>(triangles.size());
    std::vector<double> areas(T), smallest_alt(T), aspect(T);
    parallel_ranges(T, nthreads, [&](int t0, int t1, int) {
        for (int ti = t0; ti < t1; ++ti) {
            Tri& tri = triangles[ti];
            const int a = tri.vertex_ids[0], b = tri.vertex_ids[1], c = tri.vertex_ids[2];
            const double s1[3] = {P(b, 0) - P(a, 0), P(b, 1) - P(a, 1), P(b, 2) - P(a, 2)};
            const double s2[3] = {P(c, 0) - P(a, 0), P(c, 1) - P(a, 1), P(c, 2) - P(a, 2)};
            const double cx = 0.5 * (s1[1] * s2[2] - s1[2] * s2[1]);
            const double cy = 0.5 * (s1[2] * s2[0] - s1[0] * s2[2]);
            const double cz = 0.5 * (s1[0] * s2[1] - s1[1] * s2[0]);
            tri.ref_area = norm3(cx, cy, cz);
            areas[ti] = tri.ref_area;
            const double l1 = norm3(P(b, 0) - P(a, 0), P(b, 1) - P(a, 1), P(b, 2) - P(a, 2));
            const double l2 = norm3(P(c, 0) - P(a, 0), P(c, 1) - P(a, 1), P(c, 2) - P(a, 2));
            const double l3 = norm3(P(c, 0) - P(b, 0), P(c, 1) - P(b, 1), P(c, 2) - P(b, 2));
            const double alt[3] = {2.0 * tri.ref_area / l1, 2.0 * tri.ref_area / l2, 2.0 * tri.ref_area / l3};
            const double lo = *std::min_element(alt, alt + 3), hi = *std::max_element(alt, alt + 3);
            smallest_alt[ti] = lo;
            aspect[ti] = lo / hi;
            for (int k = 0; k < 3; ++k)
                tri.ref_centroid[k] = (P(a, k) + P(b, k) + P(c, k)) / 3.0;
        }
    });
    stuff.total_ref_area = kahan_sum(areas);
    size_t smallest_tri = 0, worst_tri = 0;
    stuff.approx_min_tri_size = vmin(smallest_alt, &smallest_tri);
    double worst = vmin(aspect, &worst_tri);
    log << "Approx smallest tri linear size = " << stuff.approx_min_tri_size << " (tri " << smallest_tri << ")"
        << std::endl;
    log << "Worst tri aspect ratio = " << worst << " (tri " << worst_tri
        << "). Around 0 is bad, 1 would be perfection." << std::endl;
}


void log_patch_retries(Log& log, int num_interior_retries) {
    log << "\nNumber of non-boundary triangles that had to search through \n"
        << "multiple possible patch options to find one \nsatisfying the condition number "
        << "criterion was " << num_interior_retries << ", \nwhich should not be a large proportion of the mesh's "
        << "triangles." << std::endl;
}

// source_files/set_up_patch_fitting.cpp:48-305.  For each triangle, the
// three extra patch nodes are the nearest candidates (vertices of triangles
// incident on its vertices, nearest first) whose 6x6 quadratic-fit matrix is
// invertible and well conditioned; the kept 6x3 block maps the six patch
// nodes' values to the second derivatives (xx, xy, yy) at the centroid.
void fit_patch(int t_index, const std::vector<Node>& nodes, const DMat& P, std::vector<Tri>& triangles,
               double thresh, int& num_interior_retries) {
    Tri& tri = triangles[t_index];
    std::vector<double> dists;
    std::vector<int> cands;
    for (int v = 0; v < 3; ++v)
        for (int it : nodes[tri.vertex_ids[v]].incident_tri_ids)
            for (int w = 0; w < 3; ++w) {
                int id = triangles[it].vertex_ids[w];
                bool seen = (id == tri.vertex_ids[0] || id == tri.vertex_ids[1] || id == tri.vertex_ids[2]);
                for (int c : cands) seen = seen || (c == id);
                if (!seen) {
                    dists.push_back(patch::centroid_distance(&P.v[static_cast<size_t>(id) * 3], tri.ref_centroid));
                    cands.push_back(id);
                }
            }
    if (cands.size() < 3)
        throw std::runtime_error("At least one search for patch nodes was exhausted without success (triangle " +
                                 std::to_string(tri.id) + "): fewer than 3 candidate patch nodes.");
    std::vector<size_t> order(dists.size());
    for (size_t q = 0; q < order.size(); ++q) order[q] = q;
    std::sort(order.begin(), order.end(), [&dists](const size_t& a, const size_t& b) { return dists[a] < dists[b]; });
    tri.non_vertex_patch_nodes_ids[0] = cands[order[0]];
    bool success = false;
    for (size_t p = 1; p < std::min<size_t>(4, order.size()) && !success; ++p) {
        tri.non_vertex_patch_nodes_ids[1] = cands[order[p]];
        for (size_t q = 2; q < cands.size(); ++q) {
            tri.non_vertex_patch_nodes_ids[2] = cands[order[q]];
            const int ids[6] = {tri.vertex_ids[0], tri.vertex_ids[1], tri.vertex_ids[2],
                                tri.non_vertex_patch_nodes_ids[0], tri.non_vertex_patch_nodes_ids[1],
                                tri.non_vertex_patch_nodes_ids[2]};
            double pos[6][3];
            for (int n = 0; n < 6; ++n)
                for (int c = 0; c < 3; ++c) pos[n][c] = P(ids[n], c);
            double block[6][3];
            const bool accepted = patch::try_patch(pos, tri.ref_centroid, thresh, block);
            if (!accepted) {
                if (q == 2 && !tri.is_boundary) num_interior_retries += 1;
                continue;
            }
            for (int r = 0; r < 6; ++r)
                for (int c = 0; c < 3; ++c) tri.mat_for_patch_2nd_derivs[r][c] = block[r][c];
            success = true;
            break;
        }
    }
    if (!success)
        throw std::runtime_error(
            "At least one search for patch nodes was exhausted without success (triangle " +
            std::to_string(tri.id) +
            "); all possible patch matrices in the search had a  condition number above the acceptance "
            "threshold. Try increasing this threshold. If that does not solve the issue, or causes other "
            "issues, either the patch node search will need to be extended, or you will need to use a nicer "
            "mesh. Aborting.");
}

void set_up_patch_fitting(const std::vector<Node>& nodes, const DMat& P, std::vector<Tri>& triangles,
                          const Stuff& stuff, Log& log) {
    // Triangles are independent: ranges of them in parallel threads, each
    // with its own retry count (the same choices as a serial loop).
    const int nt = setup_threads((int)triangles.size());
    std::vector<int> retries(nt, 0);
    parallel_ranges((int)triangles.size(), nt, [&](int t_begin, int t_end, int worker) {
        for (int t_index = t_begin; t_index < t_end; ++t_index)
            fit_patch(t_index, nodes, P, triangles, stuff.patch_mat_dimless_conditioning_thresh, retries[worker]);
    });
    int num_interior_retries = 0;
    for (int r : retries) num_interior_retries += r;
    log_patch_retries(log, num_interior_retries);
}

void deriv_coeffs_of(const Tri& tri, const DMat& P, double* c) {
    double vpos[3][3];
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) vpos[v][k] = P(tri.vertex_ids[v], k);
    patch::first_derivative_weights(vpos, tri.ref_centroid, c);
    for (int n = 0; n < 6; ++n)
        for (int k = 0; k < 3; ++k) c[6 + 3 * n + k] = tri.mat_for_patch_2nd_derivs[n][k];
}

// source_files/calc_deriv_mats.cpp:46-136, kept as a dense per-triangle table
// instead of the sparse num_cq x num_dofs matrix: first-derivative weights
// from the inverse of the linear-interpolation matrix, second-derivative
// weights from the patch fit.
void calc_deriv_coeffs(std::vector<double>& coeffs, const DMat& P, const std::vector<Tri>& triangles,
                       const Stuff& stuff) {
    coeffs.assign(static_cast<size_t>(stuff.num_tris) * 24, 0.0);
    parallel_ranges((int)triangles.size(), setup_threads((int)triangles.size()), [&](int b, int e, int) {
        for (int t_index = b; t_index < e; ++t_index)
            deriv_coeffs_of(triangles[t_index], P, &coeffs[static_cast<size_t>(triangles[t_index].id) * 24]);
    });
}

// source_files/calc_dof_masses.cpp:45-58: a third of each triangle's mass to
// each of its vertices (one value per node; x, y and z dofs are equal).
void calc_dof_masses(std::vector<double>& m, const std::vector<Tri>& triangles, const Stuff& stuff) {
    m.assign(stuff.num_nodes, 0.0);
    for (const auto& tri : triangles)
        for (int v = 0; v < 3; ++v) m[tri.vertex_ids[v]] += stuff.ref_density * tri.ref_area * tri.ref_thickness / 3.0;
}

// source_files/calc_char_mechanics_scales.cpp:45-73
void calc_char_mechanics_scales(const std::vector<Tri>& triangles, Stuff& stuff) {
    std::vector<double> h, mu, area;
    for (const auto& t : triangles) {
        h.push_back(t.ref_thickness);
        mu.push_back(t.ref_shear_modulus);
        area.push_back(t.ref_area);
    }
    stuff.min_ref_thickness = vmin(h);
    stuff.min_ref_shear_modulus = vmin(mu);
    stuff.char_flexural_rigidity = (1.0 / 6.0) * stuff.min_ref_shear_modulus * stuff.min_ref_thickness *
                                   stuff.min_ref_thickness * stuff.min_ref_thickness / (1.0 - stuff.def_poisson_ratio);
    stuff.char_force_scale = stuff.min_ref_shear_modulus * stuff.approx_min_tri_size * stuff.min_ref_thickness;
    stuff.char_speed_scale = std::sqrt(stuff.min_ref_shear_modulus / stuff.ref_density);
    stuff.char_stretch_energy_density_scale = stuff.min_ref_shear_modulus * stuff.min_ref_thickness;
    stuff.char_stretch_energy_scale = stuff.char_stretch_energy_density_scale * kahan_sum(area);
}

// source_files/calc_long_timescales.cpp:40-61
void calc_long_timescales(Stuff& stuff, Log& log) {
    const double pi = 3.14159265358979323846;
    const double k = 2.0 * pi / stuff.sample_char_length;
    stuff.stretch_long_time = 2.0 * pi * std::sqrt(stuff.ref_density / stuff.min_ref_shear_modulus) / k;
    stuff.bend_long_time =
        2.0 * pi * std::sqrt(stuff.ref_density * stuff.min_ref_thickness / stuff.char_flexural_rigidity) / (k * k);
    stuff.char_long_time = stuff.stretch_long_time > stuff.bend_long_time ? stuff.stretch_long_time : stuff.bend_long_time;
    log << "The long characteristic time = " << stuff.char_long_time << std::endl;
}

// source_files/calc_damping_factor.cpp:42-58
void calc_damping_factor(double prefactor, Stuff& stuff, Log& log) {
    const double pi = 3.14159265358979323846;
    const double k = 2.0 * pi / stuff.sample_char_length;
    const double scale = 2.0 * std::sqrt(stuff.char_flexural_rigidity * stuff.ref_density * stuff.min_ref_thickness *
                                         stuff.min_ref_thickness * stuff.min_ref_thickness) *
                         k * k;
    stuff.damping_factor = prefactor * scale;
    log << "Numerical Damping Coefficient = " << stuff.damping_factor << std::endl;
}

// source_files/calc_timestep.cpp:41-73
void calc_timestep(Stuff& stuff, Log& log) {
    const double pi = 3.14159265358979323846;
    double st = 0.185 * stuff.timestep_prefactor * std::sqrt(stuff.ref_density / stuff.min_ref_shear_modulus) *
                stuff.approx_min_tri_size;
    double bt = stuff.timestep_prefactor *
                std::sqrt(stuff.ref_density * stuff.min_ref_thickness / stuff.char_flexural_rigidity) *
                stuff.approx_min_tri_size * stuff.approx_min_tri_size / (2 * pi);
    log << "Short stretching and bending timescales: " << st << ", " << bt << std::endl;
    if (stuff.using_gradient_descent_dynamics) {
        st = 0.185 * stuff.timestep_prefactor *
             (stuff.damping_factor / (stuff.min_ref_shear_modulus * stuff.min_ref_thickness * stuff.min_ref_thickness)) *
             stuff.approx_min_tri_size * stuff.approx_min_tri_size / (2.0 * pi);
        bt = stuff.timestep_prefactor * (stuff.damping_factor / (stuff.char_flexural_rigidity * stuff.min_ref_thickness)) *
             stuff.approx_min_tri_size * stuff.approx_min_tri_size * stuff.approx_min_tri_size *
             stuff.approx_min_tri_size / (2.0 * pi * 2.0 * pi * 2.0 * pi);
    }
    if (st < bt) {
        stuff.timestep = st;
        log << "Time step = " << stuff.timestep << ", set based on stretching rather than bending." << std::endl;
    } else {
        stuff.timestep = bt;
        log << "Time step = " << stuff.timestep << ", set based on bending rather than stretching." << std::endl;
    }
}

// source_files/calc_steps_between_outputs.cpp:40-66
void calc_steps_between_outputs(Stuff& stuff, Log& log) {
    if (stuff.outputs_per_char_long_time < 0.0) {
        stuff.steps_between_outputs = -1;
        stuff.output_regularly = false;
        log << "The setting printouts_per_char_long_time < 0, so regular printouts have been turned off completely."
            << std::endl;
    } else {
        if (stuff.outputs_per_char_long_time < 1.0)
            throw std::runtime_error(
                "Error: To avoid potential divide-by-zero problems we do NOT allow stuff.printouts_per_char_long_time "
                "to lie in [0.0, 1.0). This is overkill somewhat, and could be relaxed if need be.");
        stuff.output_regularly = true;
        stuff.steps_between_outputs =
            std::lround(stuff.char_long_time / (stuff.timestep * stuff.outputs_per_char_long_time)) + 1;
    }
    if (stuff.using_gradient_descent_dynamics) stuff.steps_between_outputs = 1000;
}

// source_files/calc_dialling_procedure_params.cpp:52-80
void calc_dialling_procedure_params(Stuff& stuff, Log& log) {
    if (stuff.dial_factors_to_hold_at_spacing <= 0 || stuff.dial_phase_time_prefactor < 0)
        throw std::runtime_error(
            "\nstuff.step_between_dial_factors_to_hold_at and stuff.dial_phase_time must "
            "be >0 and >=0 respectively, and they aren't currently. Aborting.");
    stuff.dial_phase_time = stuff.dial_phase_time_prefactor * stuff.char_long_time;
    stuff.timesteps_per_dial_phase = std::lround(stuff.dial_phase_time / stuff.timestep);
    log << "Duration of each dialling phase = " << stuff.dial_phase_time << " which is "
        << stuff.timesteps_per_dial_phase << " timesteps." << std::endl;
    stuff.timesteps_between_equil_checks =
        std::lround(stuff.time_between_equil_checks_prefactor * stuff.dial_phase_time / stuff.timestep);
    if (stuff.timesteps_per_dial_phase <= 0)
        throw std::runtime_error("Error: the dialling phase is shorter than one timestep.");
}

// source_files/perturb_node_positions_with_noise.cpp:45-62: uniform noise of
// half-width 0.001 * approx_min_tri_size on every coordinate, from a
// minimal-standard LCG seeded with 123456.
void perturb_node_positions_with_noise(DMat& P, const Stuff& stuff) {
    std::minstd_rand engine(123456);
    std::uniform_real_distribution<double> distr(-stuff.approx_min_tri_size * 0.001, stuff.approx_min_tri_size * 0.001);
    for (int n = 0; n < stuff.num_nodes; ++n)
        for (int c = 0; c < 3; ++c) P(n, c) += distr(engine);
}

// source_files/initialize_glass_slides.cpp:27-48
void initialize_glass_slides(const DMat& P, Stuff& stuff) {
    if (stuff.using_initial_glass_slide_z_coords_from_settings_file) {
        stuff.upper_slide_z_coord = stuff.initial_upper_slide_z_coord;
        stuff.lower_slide_z_coord = stuff.initial_lower_slide_z_coord;
    } else {
        std::vector<double> z;
        for (int n = 0; n < stuff.num_nodes; ++n) z.push_back(P(n, 2));
        stuff.upper_slide_z_coord = vmax(z);
        stuff.lower_slide_z_coord = vmin(z);
    }
}

}  // namespace msb
