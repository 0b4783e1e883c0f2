// Legacy-VTK input and output in the reference's strict layout.
//   input  : source_files/read_vtk_data.cpp:65-371 (mesh + programmed fields)
//            and :380-445 (ansatz, an output file of an earlier run)
//   output : source_files/write_output.cpp:46-170 (also the restart format)
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>

#include "host.hpp"

namespace msb {

namespace {

// The whole file in memory, read with the std::istream operations the
// reference's reader uses (operator>> for words, int, bool, double;
// ignore(n, delim); ignore(1)) and their "C"-locale semantics: whitespace
// is skipped before a formatted read; a read that finds nothing it can
// convert sets `fail`, after which every operation does nothing; running
// into the end sets `eof`; numbers follow num_get's grammar (an int is
// [+-]digits, overflow saturates and fails; a double is
// [+-]digits[.digits][(e|E)[+-]digits] converted by strtod, out of range
// fails; a bool is an integer 0 or 1, anything else fails and reads true).
// Parsing from memory instead of through a stream is several times faster on
// files of millions of lines.
class Cursor {
public:
    Cursor() = default;
    // The window [p, n) of d.
    Cursor(const char* d, size_t n, size_t p) : d_(d), n_(n), p_(p) {}
    bool fail() const { return fail_; }
    bool eof() const { return eof_; }
    size_t pos() const { return p_; }

    // ignore(max, delim): up to and including the next delim, or to the end.
    void ignore_past(char delim) {
        if (!good()) {
            fail_ = true;
            return;
        }
        const void* q = p_ < n_ ? std::memchr(d_ + p_, delim, n_ - p_) : nullptr;
        if (!q) {
            p_ = n_;
            eof_ = true;
        } else {
            p_ = static_cast<size_t>(static_cast<const char*>(q) - d_) + 1;
        }
    }
    // ignore(1)
    void ignore_one() {
        if (!good()) {
            fail_ = true;
            return;
        }
        if (p_ < n_) ++p_;
        else eof_ = true;
    }
    Cursor& operator>>(std::string& w) {
        if (!begin()) return *this;
        const size_t q0 = p_;
        while (p_ < n_ && !is_space(d_[p_])) ++p_;
        if (p_ == n_) eof_ = true;
        w.assign(d_ + q0, p_ - q0);
        return *this;
    }
    Cursor& operator>>(int& v) {
        long long x = 0;
        if (!read_integer(x)) {
            v = 0;
            return *this;
        }
        if (x > INT_MAX || x < INT_MIN) {
            v = x > 0 ? INT_MAX : INT_MIN;
            fail_ = true;
        } else {
            v = static_cast<int>(x);
        }
        return *this;
    }
    Cursor& operator>>(bool& v) {
        long long x = -1;
        read_integer(x);
        if (x == 0 || x == 1) {
            v = x == 1;
        } else {
            v = true;
            fail_ = true;
        }
        return *this;
    }
    Cursor& operator>>(double& v) {
        if (!begin()) return *this;
        const size_t q0 = p_;
        size_t q = p_;
        auto digits = [&]() {
            while (q < n_ && d_[q] >= '0' && d_[q] <= '9') ++q;
        };
        if (q < n_ && (d_[q] == '+' || d_[q] == '-')) ++q;
        digits();
        if (q < n_ && d_[q] == '.') {
            ++q;
            digits();
        }
        if (q < n_ && (d_[q] == 'e' || d_[q] == 'E')) {
            ++q;
            if (q < n_ && (d_[q] == '+' || d_[q] == '-')) ++q;
            digits();
        }
        p_ = q;
        if (p_ == n_) eof_ = true;
        char buf[128];
        std::string big;
        const char* tok = buf;
        const size_t len = q - q0;
        if (len < sizeof buf) {
            std::memcpy(buf, d_ + q0, len);
            buf[len] = 0;
        } else {
            big.assign(d_ + q0, len);
            tok = big.c_str();
        }
        char* end = nullptr;
        const double x = len ? std::strtod(tok, &end) : 0.0;
        if (len == 0 || end != tok + len) {
            v = 0.0;
            fail_ = true;
        } else if (std::isinf(x)) {
            v = x > 0 ? std::numeric_limits<double>::max() : -std::numeric_limits<double>::max();
            fail_ = true;
        } else {
            v = x;
        }
        return *this;
    }

protected:
    static bool is_space(char c) {
        return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
    }
    bool good() const { return !fail_ && !eof_; }
    // The sentry of a formatted read: fails when not good, else skips
    // whitespace; false (fail and eof set) when only whitespace is left.
    bool begin() {
        if (!good()) {
            fail_ = true;
            return false;
        }
        while (p_ < n_ && is_space(d_[p_])) ++p_;
        if (p_ == n_) {
            eof_ = fail_ = true;
            return false;
        }
        return true;
    }
    bool read_integer(long long& x) {
        if (!begin()) return false;
        size_t q = p_;
        bool neg = false;
        if (d_[q] == '+' || d_[q] == '-') {
            neg = d_[q] == '-';
            ++q;
        }
        const size_t d0 = q;
        unsigned long long acc = 0;
        bool over = false;
        while (q < n_ && d_[q] >= '0' && d_[q] <= '9') {
            const unsigned dg = static_cast<unsigned>(d_[q] - '0');
            if (acc > (ULLONG_MAX - dg) / 10) over = true;
            else acc = acc * 10 + dg;
            ++q;
        }
        p_ = q;
        if (p_ == n_) eof_ = true;
        if (q == d0) {
            x = 0;
            fail_ = true;
            return false;
        }
        if (over || acc > static_cast<unsigned long long>(LLONG_MAX)) {
            x = neg ? LLONG_MIN : LLONG_MAX;
            return true;
        }
        x = neg ? -static_cast<long long>(acc) : static_cast<long long>(acc);
        return true;
    }

    const char* d_ = nullptr;
    size_t n_ = 0, p_ = 0;
    bool fail_ = false, eof_ = false;
};

// The whole file with a cursor over it.
class Scan : public Cursor {
public:
    bool open(const std::string& path) {
        std::ifstream f(path, std::ios::binary);
        if (!f) return false;
        f.seekg(0, std::ios::end);
        const std::streamoff n = f.tellg();
        if (n < 0) return false;
        f.seekg(0, std::ios::beg);
        s_.resize(static_cast<size_t>(n));
        if (n > 0 && !f.read(&s_[0], n)) return false;
        d_ = s_.data();
        n_ = s_.size();
        p_ = 0;
        return true;
    }

    // The next `count` lines, each read by line(cursor, i) with a cursor
    // limited to that line (without its newline), in parallel; afterwards
    // the position is past the last line, as after reading each line and
    // ignore_past('\n').  Returns false, with nothing moved, unless every
    // line is there and reads without a failure, i.e. unless the stream
    // reads of those lines would have found the same values on the same
    // lines; the caller then reads the lines one after another instead.
    template <typename F>
    bool lines_in_parallel(int count, F line) {
        if (!good() || count <= 0) return false;
        std::vector<size_t> start(static_cast<size_t>(count) + 1);
        size_t q = p_;
        for (int i = 0; i < count; ++i) {
            start[i] = q;
            const void* nl = q < n_ ? std::memchr(d_ + q, '\n', n_ - q) : nullptr;
            if (!nl) return false;
            q = static_cast<size_t>(static_cast<const char*>(nl) - d_) + 1;
        }
        start[count] = q;
        const int threads = setup_threads(count);
        std::vector<char> ok(threads, 1);
        parallel_ranges(count, threads, [&](int a, int b, int w) {
            for (int i = a; i < b && ok[w]; ++i) {
                Cursor c(d_, start[i + 1] - 1, start[i]);
                line(c, i);
                if (c.fail()) ok[w] = 0;
            }
        });
        for (char k : ok)
            if (!k) return false;
        p_ = q;
        return true;
    }

private:
    std::string s_;
};

void expect_word(Cursor& in, const char* word, const std::string& msg) {
    std::string temp;
    in >> temp;
    if (temp != word) throw std::runtime_error(msg);
}

}  // namespace

void read_vtk_data(std::vector<Node>& nodes, DMat& node_positions,
                   std::vector<std::array<double, 3>>& ansatz_node_positions, std::vector<Tri>& triangles,
                   DMat& abar_info, DMat& bbar_info, Stuff& stuff, double& dial_factor_to_start_from, Log& log) {
    log << "Beginning reading of reference data file." << std::endl;
    Scan in;
    if (!in.open(stuff.ref_data_filepath)) throw std::runtime_error("Error: Problem opening reference data file.");
    for (int i = 0; i < 4; ++i) in.ignore_past('\n');
    in.ignore_past(' ');
    stuff.num_nodes = 0;
    in >> stuff.num_nodes;
    if (!(stuff.num_nodes > 0))
        throw std::runtime_error("Error: Problem with (or before) line giving number of nodes in reference data file.");
    nodes.assign(stuff.num_nodes, Node());
    node_positions.resize(stuff.num_nodes, 3);
    in.ignore_past('\n');
    // The big blocks read their lines in parallel when they are well formed
    // (Scan::lines_in_parallel), else one after another as the reference does.
    for (int n = 0; n < stuff.num_nodes; ++n) nodes[n].id = n;
    if (!in.lines_in_parallel(stuff.num_nodes, [&](Cursor& c, int n) {
            c >> node_positions(n, 0) >> node_positions(n, 1) >> node_positions(n, 2);
        }))
        for (int n = 0; n < stuff.num_nodes; ++n) {
            in >> node_positions(n, 0) >> node_positions(n, 1) >> node_positions(n, 2);
            in.ignore_past('\n');
        }
    expect_word(in, "POLYGONS",
                "Error: Problem with reference data file, at or before 'POLYGONS' line. E.g. may have provided or "
                "stated wrong number of nodes.");
    stuff.num_tris = 0;
    in >> stuff.num_tris;
    if (!(stuff.num_tris > 0))
        throw std::runtime_error("Error: Problem with line giving number of triangles in reference data file.");
    triangles.assign(stuff.num_tris, Tri());
    in.ignore_past('\n');
    for (int t = 0; t < stuff.num_tris; ++t) triangles[t].id = t;
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) {
            c.ignore_one();
            c >> triangles[t].vertex_ids[0] >> triangles[t].vertex_ids[1] >> triangles[t].vertex_ids[2];
        }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            in.ignore_one();
            in >> triangles[t].vertex_ids[0] >> triangles[t].vertex_ids[1] >> triangles[t].vertex_ids[2];
            in.ignore_past('\n');
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
    in.ignore_past('\n');
    in.ignore_past('\n');
    expect_word(in, "abar_info", "Error: Problem with reference data file, at or before an abar_info line.");
    int ka = 0;
    in >> ka;
    if (ka <= 0) throw std::runtime_error("Error: Problem with reference data file, at or before an abar_info line.");
    abar_info.resize(stuff.num_tris, ka);
    in.ignore_past('\n');
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) {
            for (int p = 0; p < ka; ++p) c >> abar_info(t, p);
        }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            for (int p = 0; p < ka; ++p) in >> abar_info(t, p);
            in.ignore_past('\n');
        }
    expect_word(in, "bbar_info",
                "Error: Problem with reference data file, at or before a bbar_info line. E.g. you may have provided "
                "wrong number of abar_info lines.");
    int kb = 0;
    in >> kb;
    if (kb <= 0)
        throw std::runtime_error("Error: Problem with reference data file, at or before a bbar_info line.");
    bbar_info.resize(stuff.num_tris, kb);
    in.ignore_past('\n');
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) {
            for (int p = 0; p < kb; ++p) c >> bbar_info(t, p);
        }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            for (int p = 0; p < kb; ++p) in >> bbar_info(t, p);
            in.ignore_past('\n');
        }
    expect_word(in, "ref_thicknesses",
                "Error: Problem with reference data file, at or before a ref_thicknesses line. E.g. you may have "
                "provided wrong number of bbar_info lines.");
    in.ignore_past('\n');
    if (stuff.ref_thickness_if_uniform > 0)
        log << "Using uniform ref_thickness = " << stuff.ref_thickness_if_uniform << std::endl;
    else
        log << "Using non-uniform ref_thickness from vtk file. " << std::endl;
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) { c >> triangles[t].ref_thickness; }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            in >> triangles[t].ref_thickness;
            in.ignore_past('\n');
        }
    if (stuff.ref_thickness_if_uniform > 0)
        for (auto& tri : triangles) tri.ref_thickness = stuff.ref_thickness_if_uniform;
    expect_word(in, "ref_shear_moduli",
                "Error: Problem with reference data file, at or before a ref_shear_moduli line. E.g. you may have "
                "provided wrong number of ref_thicknesses lines.");
    in.ignore_past('\n');
    if (stuff.ref_shear_modulus_if_uniform > 0)
        log << "Using uniform ref_shear_modulus = " << stuff.ref_shear_modulus_if_uniform << std::endl;
    else
        log << "Using non-uniform ref_shear_modulus from vtk file. " << std::endl;
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) { c >> triangles[t].ref_shear_modulus; }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            in >> triangles[t].ref_shear_modulus;
            in.ignore_past('\n');
        }
    if (stuff.ref_shear_modulus_if_uniform > 0)
        for (auto& tri : triangles) tri.ref_shear_modulus = stuff.ref_shear_modulus_if_uniform;
    expect_word(in, "tri_tags", "Error: Problem with reference data file, at or before tri_tags.");
    in.ignore_past('\n');
    if (!in.lines_in_parallel(stuff.num_tris, [&](Cursor& c, int t) { c >> triangles[t].tag; }))
        for (int t = 0; t < stuff.num_tris; ++t) {
            in >> triangles[t].tag;
            in.ignore_past('\n');
        }
    expect_word(in, "POINT_DATA",
                "Error: Problem with reference data file, at or before 'POINT_DATA'. E.g. you may have provided "
                "wrong number of ref_thickness values.");
    in.ignore_past('\n');
    in.ignore_past('\n');
    expect_word(in, "constraint_indicators",
                "Error: Problem with reference data file, at or before constraint_indicators.");
    in.ignore_past('\n');
    if (!in.lines_in_parallel(stuff.num_nodes, [&](Cursor& c, int n) { c >> nodes[n].is_constrained; }))
        for (int n = 0; n < stuff.num_nodes; ++n) {
            in >> nodes[n].is_constrained;
            in.ignore_past('\n');
        }
    expect_word(in, "node_tags", "Error: Problem with reference data file, at or before node_tags.");
    in.ignore_past('\n');
    if (!in.lines_in_parallel(stuff.num_nodes, [&](Cursor& c, int n) { c >> nodes[n].tag; }))
        for (int n = 0; n < stuff.num_nodes; ++n) {
            in >> nodes[n].tag;
            in.ignore_past('\n');
        }
    if (in.fail())
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
        Scan an;
        if (!an.open(stuff.ansatz_filepath)) throw std::runtime_error("Error: Problem opening ansatz data file.");
        an.ignore_past('\n');
        an.ignore_past(' ');
        an.ignore_past(' ');
        dial_factor_to_start_from = -1.0;
        an >> dial_factor_to_start_from;
        an.ignore_past('\n');
        if (!(0 <= dial_factor_to_start_from) || !(dial_factor_to_start_from <= 1))
            throw std::runtime_error(
                "Error: Problem reading ansatz data file. Remember it must have exactly the correct format.");
        an.ignore_past('\n');
        an.ignore_past('\n');
        an.ignore_past(' ');
        int n_ans = -1;
        an >> n_ans;
        if (n_ans != stuff.num_nodes)
            throw std::runtime_error(
                "Error: Problem with (or before) line giving number of nodes in ansatz data file. "
                "E.g. you may have supplied ansatz and ref data files with inconsistent numbers of nodes.");
        an.ignore_past('\n');
        ansatz_node_positions.assign(stuff.num_nodes, {0.0, 0.0, 0.0});
        if (!an.lines_in_parallel(stuff.num_nodes, [&](Cursor& c, int n) {
                c >> ansatz_node_positions[n][0] >> ansatz_node_positions[n][1] >> ansatz_node_positions[n][2];
            }))
            for (int n = 0; n < stuff.num_nodes; ++n) {
                an >> ansatz_node_positions[n][0] >> ansatz_node_positions[n][1] >> ansatz_node_positions[n][2];
                an.ignore_past('\n');
            }
        if (an.fail())
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
