// Settings-file reader: the reference's strict "name = value;" format
// (source_files/read_settings.cpp:47-264).  Comments start with //, all
// whitespace is ignored, and the settings must appear in a fixed order.
#include <algorithm>
#include <cctype>
#include <ctime>
#include <iomanip>
#include <sstream>

#include "host.hpp"

namespace msb {

namespace {

std::vector<size_t> positions_of(const std::string& str, char c) {
    std::vector<size_t> out;
    for (size_t i = 0; i < str.size(); ++i)
        if (str[i] == c) out.push_back(i);
    return out;
}

bool parse_bool(const std::string& s) {
    if (s == "true") return true;
    if (s == "false") return false;
    throw std::runtime_error(
        "Error: you passed a std::string to boolstring_to_bool that read neither true nor false.");
}

}  // namespace

std::string get_real_time() {
    std::time_t t = std::time(nullptr);
    std::tm tm = *std::localtime(&t);
    std::ostringstream os;
    os << std::put_time(&tm, "%Y-%m-%d %H:%M:%S");
    return os.str();
}

void read_settings(Stuff& stuff, Log& log) {
    std::ifstream f(stuff.settings_filepath);
    if (!f) throw std::runtime_error("Error: Problem opening settings file.");
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    std::replace(text.begin(), text.end(), '\r', '\n');
    text.push_back('\n');
    // Strip // comments up to and including the end of their line.
    for (;;) {
        size_t c = text.find("//");
        if (c == std::string::npos) break;
        size_t nl = text.find('\n', c);
        text.erase(c, nl - c + 1);
    }
    text.erase(std::remove_if(text.begin(), text.end(), [](unsigned char x) { return std::isspace(x); }),
               text.end());

    std::vector<size_t> eq = positions_of(text, '='), sc = positions_of(text, ';');
    if (eq.size() != sc.size())
        throw std::runtime_error(
            "Error: After removing all comments, the settings file did not have equal numbers of = and ; \n "
            "The most common mistake is to forget a semicolon.");
    for (size_t j = 0; j < eq.size(); ++j) {
        bool ok = eq[j] < sc[j] && (j == 0 || sc[j - 1] < eq[j]);
        if (!ok)
            throw std::runtime_error(
                "Error: After removing all comments, the = and ; in the settings file did not occur in the correct order.");
    }
    std::vector<std::string> names, values;
    size_t cursor = 0;
    for (size_t k = 0; k < eq.size(); ++k) {
        names.push_back(text.substr(cursor, eq[k] - cursor));
        values.push_back(text.substr(eq[k] + 1, sc[k] - eq[k] - 1));
        cursor = sc[k] + 1;
    }

    size_t j = 0;
    auto expect = [&](const char* name) -> const std::string& {
        if (j >= names.size() || names[j] != name)
            throw std::runtime_error(std::string("Error: something went wrong when reading the ") + name +
                                     " setting.");
        return values[j++];
    };
    stuff.outputs_per_char_long_time = std::stod(expect("outputs_per_char_long_time"));
    stuff.ref_thickness_if_uniform = std::stod(expect("ref_thickness_if_uniform"));
    stuff.timestep_prefactor = std::stod(expect("timestep_prefactor"));
    stuff.dialling_from_ansatz_rather_than_ref_state = parse_bool(expect("dialling_from_ansatz_rather_than_ref_state"));
    stuff.dial_factors_to_hold_at_spacing = std::stod(expect("dial_factors_to_hold_at_spacing"));
    stuff.dial_phase_time_prefactor = std::stod(expect("dial_phase_time_prefactor"));
    stuff.time_between_equil_checks_prefactor = std::stod(expect("time_between_equil_checks_prefactor"));
    stuff.damping_prefactor_1 = std::stod(expect("damping_prefactor_1"));
    stuff.damping_prefactor_2 = std::stod(expect("damping_prefactor_2"));
    stuff.num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics =
        std::stoi(expect("num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics"));
    stuff.force_to_char_force_ratio_equil_threshold = std::stod(expect("force_to_char_force_ratio_equil_threshold"));
    stuff.speed_to_char_speed_ratio_equil_threshold = std::stod(expect("speed_to_char_speed_ratio_equil_threshold"));
    stuff.def_poisson_ratio = std::stod(expect("def_poisson_ratio"));
    stuff.ref_shear_modulus_if_uniform = std::stod(expect("ref_shear_modulus_if_uniform"));
    stuff.ref_density = std::stod(expect("ref_density"));
    stuff.bend_stiffening_scale_factor = std::stod(expect("bend_stiffening_scale_factor"));
    stuff.patch_mat_dimless_conditioning_thresh = std::stod(expect("patch_mat_dimless_conditioning_thresh"));
    stuff.slide_stiffness_prefactor = std::stod(expect("slide_stiffness_prefactor"));
    stuff.slide_friction_coefficent = std::stod(expect("slide_friction_coefficent"));
    stuff.slide_speed_prefactor = std::stod(expect("slide_speed_prefactor"));
    stuff.using_initial_glass_slide_z_coords_from_settings_file =
        parse_bool(expect("using_initial_glass_slide_z_coords_from_settings_file"));
    stuff.initial_upper_slide_z_coord = std::stod(expect("initial_upper_slide_z_coord"));
    stuff.initial_lower_slide_z_coord = std::stod(expect("initial_lower_slide_z_coord"));
    // Optional trailing extension; the reference stops reading before it.
    stuff.dialling_protocol = 1;
    if (j < names.size() && names[j] == "dialling_protocol") {
        stuff.dialling_protocol = std::stoi(values[j]);
        ++j;
        if (stuff.dialling_protocol < 1 || stuff.dialling_protocol > 5)
            throw std::runtime_error("Error: dialling_protocol must be one of 1, 2, 3, 4, 5.");
    }

    if (stuff.dialling_from_ansatz_rather_than_ref_state) {
        if (stuff.ansatz_file_was_given) {
            log << "You have chosen to dial abar and bbar from the a and b of the ansatz. "
                   "This will override some things: dial_factor_to_start_from will be set "
                   "to 0, and a and b will be dialled linearly from the ansatz a and b to "
                   "the final (dial_factor=1) abar and bbar."
                << std::endl;
        } else {
            throw std::runtime_error(
                "Error: You cannot use the dialling_from_ansatz_rather_than_ref_state setting if you have not "
                "supplied an ansatz file.");
        }
    }
    if (stuff.dial_factors_to_hold_at_spacing > 1.0)
        throw std::runtime_error(
            "Error: The largest permitted value of dial_factors_to_hold_at_spacing is 1.0, because dial_factor "
            "never goes above 1.0, so anything larger would be meaningless.");
    stuff.using_gradient_descent_dynamics =
        stuff.num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics > 0;
    if (stuff.using_gradient_descent_dynamics)
        log << "You have chosen to use gradient descent dynamics for "
            << stuff.num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics
            << " steps before switching to Newtonian dynamics." << std::endl;
    if (stuff.slide_stiffness_prefactor > 0.0)
        throw std::runtime_error(
            "Error: glass slides (slide_stiffness_prefactor > 0) are not supported by the GPU loop.");
}

}  // namespace msb
