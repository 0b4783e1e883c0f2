// Legacy-VTK input and output in the reference's strict layout.
//   input  : source_files/read_vtk_data.cpp:65-371 (mesh + programmed fields)
//            and :380-445 (ansatz, an output file of an earlier run)
//   output : source_files/write_output.cpp:46-170 (also the restart format)
#include <iomanip>
#include <limits>

#include "host.hpp"

namespace msb {

namespace {

constexpr std::streamsize kMax = std::numeric_limits<std::streamsize>::max();

void expect_word(std::istream& in, const char* word, const std::string& msg) {
    std::string temp;
    in >> temp;
    if (temp != word) throw std::runtime_error(msg);
}

}  // namespace

void read_vtk_data(std::vector<Node>& nodes, DMat& node_positions,
                   std::vector<std::array<double, 3>>& ansatz_node_positions, std::vector<Tri>& triangles,
                   DMat& abar_info, DMat& bbar_info, Stuff& stuff, double& dial_factor_to_start_from, Log& log) {
    log << "Beginning reading of reference data file." << std::endl;
    std::ifstream in(stuff.ref_data_filepath);
    if (!in) throw std::runtime_error("Error: Problem opening reference data file.");
    for (int i = 0; i < 4; ++i) in.ignore(kMax, '\n');
    in.ignore(kMax, ' ');
    stuff.num_nodes = 0;
    in >> stuff.num_nodes;
    if (!(stuff.num_nodes > 0))
        throw std::runtime_error("Error: Problem with (or before) line giving number of nodes in reference data file.");
    nodes.assign(stuff.num_nodes, Node());
    node_positions.resize(stuff.num_nodes, 3);
    in.ignore(kMax, '\n');
    for (int n = 0; n < stuff.num_nodes; ++n) {
        nodes[n].id = n;
        in >> node_positions(n, 0) >> node_positions(n, 1) >> node_positions(n, 2);
        in.ignore(kMax, '\n');
    }
    expect_word(in, "POLYGONS",
                "Error: Problem with reference data file, at or before 'POLYGONS' line. E.g. may have provided or "
                "stated wrong number of nodes.");
    stuff.num_tris = 0;
    in >> stuff.num_tris;
    if (!(stuff.num_tris > 0))
        throw std::runtime_error("Error: Problem with line giving number of triangles in reference data file.");
    triangles.assign(stuff.num_tris, Tri());
    in.ignore(kMax, '\n');
    for (int t = 0; t < stuff.num_tris; ++t) {
        triangles[t].id = t;
        in.ignore(1);
        in >> triangles[t].vertex_ids[0] >> triangles[t].vertex_ids[1] >> triangles[t].vertex_ids[2];
        in.ignore(kMax, '\n');
    }
    bool found_zero = false;
    for (const auto& tri : triangles)
        for (int v = 0; v < 3; ++v) found_zero |= (tri.vertex_ids[v] == 0);
    if (!found_zero)
        throw std::runtime_error(
            "Error: MorphoShell requires the triangulation you provide to use node ids starting from 0. "
            "It appears that the triangulation you provided did not do this, since it didn't contain a 0 anywhere.");
    // The reference trusts ids to be < num_nodes; a bad id would index out of
    // bounds on the device, so check it here.
    for (const auto& tri : triangles)
        for (int v = 0; v < 3; ++v)
            if (tri.vertex_ids[v] < 0 || tri.vertex_ids[v] >= stuff.num_nodes)
                throw std::runtime_error("Error: a triangle vertex id in the reference data file is out of range.");

    expect_word(in, "CELL_DATA",
                "Error: Problem with reference data file, at or before 'CELL_DATA' line. E.g. you may have provided "
                "or stated wrong number of triangles.");
    in.ignore(kMax, '\n');
    in.ignore(kMax, '\n');
    expect_word(in, "abar_info", "Error: Problem with reference data file, at or before an abar_info line.");
    int ka = 0;
    in >> ka;
    if (ka <= 0) throw std::runtime_error("Error: Problem with reference data file, at or before an abar_info line.");
    abar_info.resize(stuff.num_tris, ka);
    in.ignore(kMax, '\n');
    for (int t = 0; t < stuff.num_tris; ++t) {
        for (int p = 0; p < ka; ++p) in >> abar_info(t, p);
        in.ignore(kMax, '\n');
    }
    expect_word(in, "bbar_info",
                "Error: Problem with reference data file, at or before a bbar_info line. E.g. you may have provided "
                "wrong number of abar_info lines.");
    int kb = 0;
    in >> kb;
    if (kb <= 0)
        throw std::runtime_error("Error: Problem with reference data file, at or before a bbar_info line.");
    bbar_info.resize(stuff.num_tris, kb);
    in.ignore(kMax, '\n');
    for (int t = 0; t < stuff.num_tris; ++t) {
        for (int p = 0; p < kb; ++p) in >> bbar_info(t, p);
        in.ignore(kMax, '\n');
    }
    expect_word(in, "ref_thicknesses",
                "Error: Problem with reference data file, at or before a ref_thicknesses line. E.g. you may have "
                "provided wrong number of bbar_info lines.");
    in.ignore(kMax, '\n');
    if (stuff.ref_thickness_if_uniform > 0)
        log << "Using uniform ref_thickness = " << stuff.ref_thickness_if_uniform << std::endl;
    else
        log << "Using non-uniform ref_thickness from vtk file. " << std::endl;
    for (int t = 0; t < stuff.num_tris; ++t) {
        in >> triangles[t].ref_thickness;
        in.ignore(kMax, '\n');
        if (stuff.ref_thickness_if_uniform > 0) triangles[t].ref_thickness = stuff.ref_thickness_if_uniform;
    }
    expect_word(in, "ref_shear_moduli",
                "Error: Problem with reference data file, at or before a ref_shear_moduli line. E.g. you may have "
                "provided wrong number of ref_thicknesses lines.");
    in.ignore(kMax, '\n');
    if (stuff.ref_shear_modulus_if_uniform > 0)
        log << "Using uniform ref_shear_modulus = " << stuff.ref_shear_modulus_if_uniform << std::endl;
    else
        log << "Using non-uniform ref_shear_modulus from vtk file. " << std::endl;
    for (int t = 0; t < stuff.num_tris; ++t) {
        in >> triangles[t].ref_shear_modulus;
        in.ignore(kMax, '\n');
        if (stuff.ref_shear_modulus_if_uniform > 0) triangles[t].ref_shear_modulus = stuff.ref_shear_modulus_if_uniform;
    }
    expect_word(in, "tri_tags", "Error: Problem with reference data file, at or before tri_tags.");
    in.ignore(kMax, '\n');
    in.unsetf(std::ios_base::boolalpha);
    for (int t = 0; t < stuff.num_tris; ++t) {
        in >> triangles[t].tag;
        in.ignore(kMax, '\n');
    }
    expect_word(in, "POINT_DATA",
                "Error: Problem with reference data file, at or before 'POINT_DATA'. E.g. you may have provided "
                "wrong number of ref_thickness values.");
    in.ignore(kMax, '\n');
    in.ignore(kMax, '\n');
    expect_word(in, "constraint_indicators",
                "Error: Problem with reference data file, at or before constraint_indicators.");
    in.ignore(kMax, '\n');
    for (int n = 0; n < stuff.num_nodes; ++n) {
        in >> nodes[n].is_constrained;
        in.ignore(kMax, '\n');
    }
    expect_word(in, "node_tags", "Error: Problem with reference data file, at or before node_tags.");
    in.ignore(kMax, '\n');
    for (int n = 0; n < stuff.num_nodes; ++n) {
        in >> nodes[n].tag;
        in.ignore(kMax, '\n');
    }
    if (in.bad() || in.fail())
        throw std::runtime_error(
            "Error: Unkown problem with reference data file. One of .bad(), .fail() was true - investigate! "
            "E.g. you may not have supplied enough node indicator data in the file, so the file may have reached "
            "its end prematurely.");
    std::string rest;
    in >> rest;
    if (!in.eof())
        throw std::runtime_error(
            "Error: Did not reach end of reference data file as expected. Check that it has exactly the correct "
            "format.");
    log << "Completed reading of reference data file. Note; it is still possible that something went wrong in "
           "the process.\n"
        << std::endl;

    if (stuff.ansatz_file_was_given) {
        log << "Beginning reading of ansatz data file." << std::endl;
        std::ifstream an(stuff.ansatz_filepath);
        if (!an) throw std::runtime_error("Error: Problem opening ansatz data file.");
        an.ignore(kMax, '\n');
        an.ignore(kMax, ' ');
        an.ignore(kMax, ' ');
        dial_factor_to_start_from = -1.0;
        an >> dial_factor_to_start_from;
        an.ignore(kMax, '\n');
        if (!(0 <= dial_factor_to_start_from) || !(dial_factor_to_start_from <= 1))
            throw std::runtime_error(
                "Error: Problem reading ansatz data file. Remember it must have exactly the correct format.");
        an.ignore(kMax, '\n');
        an.ignore(kMax, '\n');
        an.ignore(kMax, ' ');
        int n_ans = -1;
        an >> n_ans;
        if (n_ans != stuff.num_nodes)
            throw std::runtime_error(
                "Error: Problem with (or before) line giving number of nodes in ansatz data file. "
                "E.g. you may have supplied ansatz and ref data files with inconsistent numbers of nodes.");
        an.ignore(kMax, '\n');
        ansatz_node_positions.assign(stuff.num_nodes, {0.0, 0.0, 0.0});
        for (int n = 0; n < stuff.num_nodes; ++n) {
            an >> ansatz_node_positions[n][0] >> ansatz_node_positions[n][1] >> ansatz_node_positions[n][2];
            an.ignore(kMax, '\n');
        }
        if (an.bad() || an.fail())
            throw std::runtime_error(
                "Error: Unkown problem with ansatz data file. One of .bad(), .fail() was true - investigate! "
                " E.g. you may not have supplied enough ansatz node positions, so the file reached its end "
                "prematurely.");
        log << "Completed reading of ansatz data file. Note, it is still possible that something went wrong in "
               "the process.\n"
            << std::endl;
    }
}

void write_output(const std::vector<double>& dofs, const std::vector<Tri>& triangles, int stepcount,
                  double dial_factor, const std::vector<double>& curvatures,
                  const std::vector<double>& energy_densities, const std::vector<double>& angle_deficits,
                  const std::vector<double>& stresses, const std::vector<double>& strains, const Stuff& stuff) {
    const int N = stuff.num_nodes, T = stuff.num_tris;
    {
        std::ofstream aux(stuff.aux_output_filepath, std::ofstream::app);
        if (stepcount == 0)
            aux << "stepcount  " << "dial_factor  " << "stuff.status  " << "upper_slide_z  " << "upper_slide_force  "
                << "lower_slide_z  " << "lower_slide_force  " << std::endl;
        aux << stepcount << "  " << dial_factor << " " << stuff.status << "  " << stuff.upper_slide_z_coord << " "
            << stuff.upper_slide_tot_vert_force << " " << stuff.lower_slide_z_coord << " "
            << stuff.lower_slide_tot_vert_force << " " << std::endl;
    }
    std::ofstream out(stuff.output_dir_path + "/stepcount_" + std::to_string(stepcount) + "_output.vtk");
    if (!out) throw std::runtime_error("Error: Problem creating or opening vtk output file.");
    out << std::scientific << std::setprecision(14) << "# vtk DataFile Version 4.2" << "\n"
        << "dial_factor = " << dial_factor << ", stepcount = " << stepcount;
    out << "\n" << "ASCII" << "\n" << "DATASET POLYDATA" << "\n" << "POINTS " << N << " double" << "\n";
    for (int n = 0; n < N; ++n) out << dofs[n] << " " << dofs[n + N] << " " << dofs[n + 2 * N] << "\n";
    out << "POLYGONS " << T << " " << 4 * T << "\n";
    for (const auto& tri : triangles)
        out << "3 " << tri.vertex_ids[0] << " " << tri.vertex_ids[1] << " " << tri.vertex_ids[2] << "\n";
    out << "CELL_DATA " << T << "\n";
    out << "SCALARS gauss_curv double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int t = 0; t < T; ++t) out << curvatures[2 * t + 0] << "\n";
    out << "SCALARS mean_curv double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int t = 0; t < T; ++t) out << curvatures[2 * t + 1] << "\n";
    out << "SCALARS dimless_stretch_energy_density double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int t = 0; t < T; ++t) out << energy_densities[2 * t + 0] / stuff.char_stretch_energy_density_scale << "\n";
    out << "SCALARS dimless_bend_energy_density double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int t = 0; t < T; ++t) out << energy_densities[2 * t + 1] / stuff.char_stretch_energy_density_scale << "\n";
    out << "SCALARS strain_measure double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int t = 0; t < T; ++t) out << strains[t] << "\n";
    out << "FIELD cauchy_stress_info 4" << "\n";
    out << "dimless_cauchy_stress_eigval_1 1 " << T << " double" << "\n";
    for (int t = 0; t < T; ++t)
        out << stresses[8 * t + 0] / (triangles[t].ref_shear_modulus * triangles[t].ref_thickness) << "\n";
    out << "cauchy_stress_eigvec_1 3 " << T << " double" << "\n";
    for (int t = 0; t < T; ++t)
        out << stresses[8 * t + 1] << " " << stresses[8 * t + 2] << " " << stresses[8 * t + 3] << "\n";
    out << "dimless_cauchy_stress_eigval_2 1 " << T << " double" << "\n";
    for (int t = 0; t < T; ++t)
        out << stresses[8 * t + 4] / (triangles[t].ref_shear_modulus * triangles[t].ref_thickness) << "\n";
    out << "cauchy_stress_eigvec_2 3 " << T << " double" << "\n";
    for (int t = 0; t < T; ++t)
        out << stresses[8 * t + 5] << " " << stresses[8 * t + 6] << " " << stresses[8 * t + 7] << "\n";
    out << "POINT_DATA " << N << "\n";
    out << "SCALARS angleDeficit double 1" << "\n" << "LOOKUP_TABLE default" << "\n";
    for (int n = 0; n < N; ++n) out << angle_deficits[n] << "\n";
}

}  // namespace msb
