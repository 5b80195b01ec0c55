// Input-script front end: the hot-path commands of the reference's script
// grammar mapped onto shhd_config (host only, no GPU needed).
//
// Grammar, defaults, validation and error messages follow the reference's
// ParamParser (src/param_parser.cc:42-163 commands, 165-284 `model`,
// 287-339 `fix`, 551-639 nonlinear / noise, 641-769 forces, 771-805
// validate_configuration) and the model styles it dispatches to
// (model_free_energy_phi4_style.h, model_free_energy_quadratic_style.h,
// model_thermodynamics_registry.h:61-72, model_transport_coefficient_registry.h:77-143).
// `set`, `measure`, `thermo`, `restart` and `run` do not shape the step and
// are accepted without interpretation.
#include <cctype>
#include <cmath>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/shhd_b200.h"

namespace {

using Tokens = std::vector<std::string>;

struct ParseState {
    shhd_config cfg{};
    int dealias = 0;          // 0 none, 1 three halves, 2 two
    bool has_transport = false;
    bool has_free_energy = false;
    std::string free_energy_type;
    bool has_thermo = false;
    bool commands_started = false;
    std::string time_evolution = "srk3/compressible";
    std::vector<std::string> sine_ids;
    std::vector<std::string> gradient_ids;
};

bool parse_on_off(const std::string& v, const std::string& ctx) {
    if (v == "on") return true;
    if (v == "off") return false;
    throw std::runtime_error(ctx + " expects on|off");
}

int parse_xy(const std::string& v, const std::string& ctx) {
    if (v == "x" || v == "0") return 0;
    if (v == "y" || v == "1") return 1;
    throw std::runtime_error(ctx + " must be x|y|0|1.");
}

bool is_quiescent(const std::string& t) { return t == "euler/quiescent" || t == "srk3/quiescent"; }

int compute_grid_size(int active, int rule) {
    if (active <= 0) throw std::runtime_error("grid size must be positive.");
    if (rule == 0) return active;
    if (rule == 1) {
        if (active % 2 != 0) throw std::runtime_error("3/2 dealiasing requires even active grid size.");
        return 3 * active / 2;
    }
    return 2 * active;
}

void update_grid(ParseState& s) {
    s.cfg.nx = compute_grid_size(s.cfg.active_nx, s.dealias);
    s.cfg.ny = compute_grid_size(s.cfg.active_ny, s.dealias);
}

// "<prefix>[<digits>]" -> index
bool indexed_key(const std::string& key, const std::string& prefix, int& idx) {
    const std::string head = prefix + "[";
    if (key.size() <= head.size() + 1 || key.back() != ']' || key.rfind(head, 0) != 0) return false;
    for (std::size_t i = head.size(); i < key.size() - 1; ++i)
        if (!std::isdigit(static_cast<unsigned char>(key[i]))) return false;
    idx = std::stoi(key.substr(head.size(), key.size() - head.size() - 1));
    return true;
}

// "M[<digits>,<digits>]"
bool mobility_key(const std::string& key, int& row, int& col) {
    if (key.size() < 6 || key[0] != 'M' || key[1] != '[' || key.back() != ']') return false;
    const std::size_t comma = key.find(',', 2);
    if (comma == std::string::npos || comma + 1 >= key.size() - 1) return false;
    for (std::size_t i = 2; i < comma; ++i) if (!std::isdigit(static_cast<unsigned char>(key[i]))) return false;
    for (std::size_t i = comma + 1; i < key.size() - 1; ++i) if (!std::isdigit(static_cast<unsigned char>(key[i]))) return false;
    row = std::stoi(key.substr(2, comma - 2));
    col = std::stoi(key.substr(comma + 1, key.size() - comma - 2));
    return true;
}

void parse_model(ParseState& s, const Tokens& t) {
    if (t.size() < 3)
        throw std::runtime_error("model syntax: model <thermo|transport> <type> [args...] | model <thermo|transport> coeff <args...>");
    const std::string& category = t[1];
    const std::string& action = t[2];
    shhd_config& c = s.cfg;
    const int nop = c.num_order_parameters;
    std::vector<std::pair<std::string, std::string>> kv;
    for (std::size_t i = 3; i < t.size(); i += 2) {
        if (i + 1 >= t.size()) throw std::runtime_error("model " + category + " " + action + " arguments must be key-value pairs");
        kv.emplace_back(t[i], t[i + 1]);
    }
    if (category == "thermo") {
        if (action == "coeff") {
            if (!s.has_thermo) throw std::runtime_error("model thermo coeff requires model thermo <type> first");
        } else {
            if (action != "linear_eos") throw std::runtime_error("Unknown thermodynamics type: " + action);
            s.has_thermo = true;
            c.cT = 0.0;
        }
        for (const auto& p : kv) {
            if (p.first == "cT" || p.first == "sound_speed") {
                const double v = std::stod(p.second);
                if (v < 0.0) throw std::runtime_error("model thermo linear_eos requires nonnegative " + p.first + ".");
                c.cT = v;
            } else {
                throw std::runtime_error("unknown linear_eos thermodynamics coefficient: " + p.first);
            }
        }
        return;
    }
    if (category == "free_energy") {
        if (action == "coeff") {
            if (!s.has_free_energy) throw std::runtime_error("model free_energy coeff requires model free_energy <type> first");
        } else {
            // the reference's styles, then the plugin styles compiled into the library
            int plugin = 0;
            for (int id = 1; id <= shhd_free_energy_plugin_count(); ++id)
                if (action == shhd_free_energy_plugin_name(id)) plugin = id;
            if (action != "phi4" && action != "quadratic" && plugin == 0) throw std::runtime_error("Unknown free energy type: " + action);
            s.has_free_energy = true;
            s.free_energy_type = action;
            c.free_energy = action == "phi4" ? SHHD_FE_PHI4 : (action == "quadratic" ? SHHD_FE_QUADRATIC : SHHD_FE_PLUGIN);
            c.fe_plugin = plugin;
            for (int a = 0; a < SHHD_MAX_ORDER_PARAMETERS; ++a) c.mu_k0[a] = c.mu_k2[a] = c.mu_k4[a] = c.mu_u3[a] = 0.0;
            for (int k = 0; k < SHHD_MAX_FE_PARAMS; ++k)
                for (int a = 0; a < SHHD_MAX_ORDER_PARAMETERS; ++a) c.fe_param[k][a] = 0.0;
        }
        for (const auto& p : kv) {
            int idx = -1;
            const double v = std::stod(p.second);
            if (s.free_energy_type == "phi4") {
                if (indexed_key(p.first, "a", idx) || indexed_key(p.first, "b", idx) || indexed_key(p.first, "u", idx)) {
                    if (idx < 0 || idx >= nop) throw std::runtime_error("model free_energy phi4 coefficient index out of range: " + p.first);
                    if (p.first[0] == 'a') c.mu_k0[idx] = v;
                    else if (p.first[0] == 'b') c.mu_k2[idx] = v;
                    else {
                        if (v < 0.0) throw std::runtime_error("model free_energy phi4 requires nonnegative " + p.first + ".");
                        c.mu_u3[idx] = v;
                    }
                    continue;
                }
                throw std::runtime_error("unknown phi4 free energy coefficient: " + p.first);
            }
            if (s.free_energy_type == "quadratic") {
                if (indexed_key(p.first, "a", idx)) {
                    if (idx < 0 || idx >= nop) throw std::runtime_error("model free_energy quadratic coefficient index out of range: " + p.first);
                    c.mu_k0[idx] = v;
                    continue;
                }
                throw std::runtime_error("unknown quadratic free energy coefficient: " + p.first);
            }
            // plugin style: linear a[], b[] as phi4, then the style's own keys
            const std::string& st = s.free_energy_type;
            if (indexed_key(p.first, "a", idx) || indexed_key(p.first, "b", idx)) {
                if (idx < 0 || idx >= nop) throw std::runtime_error("model free_energy " + st + " coefficient index out of range: " + p.first);
                (p.first[0] == 'a' ? c.mu_k0 : c.mu_k2)[idx] = v;
                continue;
            }
            bool known = false;
            for (int k = 0; !known; ++k) {
                const char* key = shhd_free_energy_plugin_key(c.fe_plugin, k);
                if (!key) break;
                const std::string ks(key);
                if (ks.size() > 2 && ks.compare(ks.size() - 2, 2, "[]") == 0) {
                    if (!indexed_key(p.first, ks.substr(0, ks.size() - 2), idx)) continue;
                    if (idx < 0 || idx >= nop) throw std::runtime_error("model free_energy " + st + " coefficient index out of range: " + p.first);
                    c.fe_param[k][idx] = v;
                } else {
                    if (p.first != ks) continue;
                    c.fe_param[k][0] = v;
                }
                known = true;
            }
            if (!known) throw std::runtime_error("unknown " + st + " free energy coefficient: " + p.first);
        }
        return;
    }
    if (category == "transport") {
        if (action == "coeff") {
            if (!s.has_transport) throw std::runtime_error("model transport coeff requires model transport <type> first");
        } else {
            if (action != "constant") throw std::runtime_error("Unknown Transport Coefficients type: " + action);
            s.has_transport = true;
            c.eta = c.zeta = 0.0;
            for (int a = 0; a < SHHD_MAX_ORDER_PARAMETERS; ++a) c.mobility[a] = 0.0;
        }
        for (const auto& p : kv) {
            const std::string& key = p.first;
            if (key == "eta" || key == "shear_viscosity" || key == "zeta" || key == "bulk_viscosity") {
                const double v = std::stod(p.second);
                if (v < 0.0) throw std::runtime_error("model transport constant requires nonnegative " + key + ".");
                if (key == "eta" || key == "shear_viscosity") c.eta = v; else c.zeta = v;
                continue;
            }
            int row = -1, col = -1;
            if (mobility_key(key, row, col)) {
                const double v = std::stod(p.second);
                if (row < 0 || row >= nop || col < 0 || col >= nop)
                    throw std::runtime_error("model transport constant mobility index out of range: " + key);
                if (row != col) {
                    if (std::abs(v) > 0.0)
                        throw std::runtime_error("model transport constant only supports diagonal mobility; " + key + " must be zero.");
                    continue;
                }
                if (v < 0.0) throw std::runtime_error("model transport constant requires nonnegative " + key + ".");
                c.mobility[row] = v;
                continue;
            }
            throw std::runtime_error("unknown constant transport coefficient: " + key);
        }
        return;
    }
    throw std::runtime_error("unknown model category: " + category);
}

void parse_fix(ParseState& s, const Tokens& t) {
    if (t.size() < 5) throw std::runtime_error("fix syntax: fix <ID> <target> <nonlinear|noise|force/sine|force/gradient> <on|off> ...");
    if (s.commands_started) throw std::runtime_error("fix must be specified before run or measure commands");
    shhd_config& c = s.cfg;
    const int nop = c.num_order_parameters;
    const std::string& id = t[1];
    const std::string& tt = t[2];
    const std::string& type = t[3];
    const bool enabled = parse_on_off(t[4], "fix " + type);
    std::string target;
    if (tt == "momentum" || tt == "j") target = "momentum";
    else if (tt == "order_parameter" || tt == "psi") {
        if (nop <= 0) throw std::runtime_error("fix " + type + " " + tt + " requires order_parameters > 0.");
        target = "order_parameter";
    } else if (tt == "all") target = "all";
    else throw std::runtime_error("unknown fix target: " + tt);

    if (type == "nonlinear") {
        if (t.size() != 5) throw std::runtime_error("fix nonlinear syntax: fix <ID> <target> nonlinear <on|off>");
        if (target == "momentum" || target == "all") c.momentum_advection = enabled;
        if (target == "order_parameter" || target == "all") c.order_parameter_advection = enabled && nop > 0;
        return;
    }
    if (type == "noise") {
        if (!enabled && t.size() != 5) throw std::runtime_error("fix noise off syntax: fix <ID> <target> noise off");
        if (enabled) {
            if ((t.size() - 5) % 2 != 0) throw std::runtime_error("fix noise syntax: fix <ID> <target> noise on [seed <integer>] [kBT <value>]");
            for (std::size_t i = 5; i < t.size(); i += 2) {
                const std::string& key = t[i];
                const std::string& value = t[i + 1];
                if (key == "seed") { c.noise_seed = std::stoi(value); continue; }
                if (key == "kBT" || key == "temperature") {
                    c.kBT = std::stod(value);
                    if (c.kBT < 0.0) throw std::runtime_error("fix noise requires nonnegative kBT.");
                    continue;
                }
                if (key == "chi" || key == "order_parameter_chi" || key == "psi_chi") {
                    if (target == "momentum") throw std::runtime_error("fix momentum noise does not use chi.");
                    if (nop <= 0) throw std::runtime_error("fix noise chi requires order_parameters > 0.");
                    c.chi = std::stod(value);
                    if (c.chi < 0.0) throw std::runtime_error("fix noise requires nonnegative chi.");
                    continue;
                }
                throw std::runtime_error("unknown fix noise argument: " + key);
            }
        }
        if (target == "momentum" || target == "all") c.noise_momentum = enabled;
        if (target == "order_parameter" || target == "all") c.noise_order_parameter = enabled && nop > 0;
        if (is_quiescent(s.time_evolution) && c.noise_momentum) c.noise_momentum = 0;
        return;
    }
    if (type == "force/sine") {
        // a force with the same ID replaces the previous one
        for (std::size_t i = 0; i < s.sine_ids.size(); ++i)
            if (s.sine_ids[i] == id) {
                for (std::size_t k = i + 1; k < s.sine_ids.size(); ++k) c.sine_forces[k - 1] = c.sine_forces[k];
                s.sine_ids.erase(s.sine_ids.begin() + static_cast<long>(i));
                --c.n_sine_forces;
                break;
            }
        if (!enabled) {
            if (t.size() != 5) throw std::runtime_error("fix force/sine off syntax: fix <ID> <target> force/sine off");
            return;
        }
        if (target == "all") throw std::runtime_error("fix force/sine does not support target all.");
        if ((t.size() - 5) % 2 != 0) throw std::runtime_error("fix force/sine arguments must be key-value pairs.");
        shhd_sine_force f{};
        f.target = target == "momentum" ? 0 : 1;
        f.component = -1; f.axis = -1; f.nk = 1;
        bool hc = false, ha = false, hn = false, hamp = false;
        for (std::size_t i = 5; i < t.size(); i += 2) {
            const std::string& key = t[i];
            const std::string& value = t[i + 1];
            if (key == "component") {
                if (f.target == 0) f.component = parse_xy(value, "fix momentum force/sine component");
                else {
                    f.component = std::stoi(value);
                    if (f.component < 0 || f.component >= nop)
                        throw std::runtime_error("fix order_parameter force/sine: order-parameter index out of range: " + value);
                }
                hc = true;
            } else if (key == "axis") { f.axis = parse_xy(value, "fix force/sine axis"); ha = true; }
            else if (key == "nk") { f.nk = std::stoi(value); hn = true; }
            else if (key == "amplitude") { f.amplitude = std::stod(value); hamp = true; }
            else throw std::runtime_error("unknown fix force/sine argument: " + key);
        }
        if (!hc || !ha || !hn || !hamp) throw std::runtime_error("fix force/sine requires component, axis, nk, and amplitude.");
        if (f.nk <= 0) throw std::runtime_error("fix force/sine requires nk > 0.");
        const int active = f.axis == 0 ? c.active_nx : c.active_ny;
        if (f.nk >= active / 2) throw std::runtime_error("fix force/sine requires nk < active_N_axis/2.");
        if (c.n_sine_forces >= SHHD_MAX_FORCES) throw std::runtime_error("too many force/sine fixes");
        c.sine_forces[c.n_sine_forces++] = f;
        s.sine_ids.push_back(id);
        return;
    }
    if (type == "force/gradient") {
        for (std::size_t i = 0; i < s.gradient_ids.size(); ++i)
            if (s.gradient_ids[i] == id) {
                for (std::size_t k = i + 1; k < s.gradient_ids.size(); ++k) c.gradient_forces[k - 1] = c.gradient_forces[k];
                s.gradient_ids.erase(s.gradient_ids.begin() + static_cast<long>(i));
                --c.n_gradient_forces;
                break;
            }
        if (!enabled) {
            if (t.size() != 5) throw std::runtime_error("fix force/gradient off syntax: fix <ID> <target> force/gradient off");
            return;
        }
        if (target != "order_parameter") throw std::runtime_error("fix force/gradient only supports target order_parameter.");
        if ((t.size() - 5) % 2 != 0) throw std::runtime_error("fix force/gradient arguments must be key-value pairs.");
        shhd_gradient_force f{};
        f.component = -1; f.direction = -1;
        bool hc = false, hd = false, ha = false;
        for (std::size_t i = 5; i < t.size(); i += 2) {
            const std::string& key = t[i];
            const std::string& value = t[i + 1];
            if (key == "component") {
                f.component = std::stoi(value);
                if (f.component < 0 || f.component >= nop)
                    throw std::runtime_error("fix order_parameter force/gradient: order-parameter index out of range: " + value);
                hc = true;
            } else if (key == "direction") { f.direction = parse_xy(value, "fix force/gradient direction"); hd = true; }
            else if (key == "amplitude") { f.amplitude = std::stod(value); ha = true; }
            else throw std::runtime_error("unknown fix force/gradient argument: " + key);
        }
        if (!hc || !hd || !ha) throw std::runtime_error("fix force/gradient requires component, direction, and amplitude.");
        if (c.n_gradient_forces >= SHHD_MAX_FORCES) throw std::runtime_error("too many force/gradient fixes");
        c.gradient_forces[c.n_gradient_forces++] = f;
        s.gradient_ids.push_back(id);
        return;
    }
    throw std::runtime_error("unknown fix style: " + type);
}

void execute(ParseState& s, const Tokens& t) {
    if (t.empty()) return;
    const std::string& cmd = t[0];
    shhd_config& c = s.cfg;
    if (cmd == "dimension") {
        if (t.size() < 2) throw std::runtime_error("dimension syntax: dimension <num>");
        if (std::stoi(t[1]) != 2) throw std::runtime_error("This solver only supports dimension 2.");
    } else if (cmd == "order_parameters" || cmd == "order_parameter") {
        if (t.size() != 2) throw std::runtime_error("order_parameters syntax: order_parameters <num>");
        c.num_order_parameters = std::stoi(t[1]);
        if (c.num_order_parameters < 0) throw std::runtime_error("order_parameters must be nonnegative.");
        if (c.num_order_parameters > SHHD_MAX_ORDER_PARAMETERS)
            throw std::runtime_error("order_parameters above " + std::to_string(SHHD_MAX_ORDER_PARAMETERS) + " are not supported by this engine.");
    } else if (cmd == "boundary") {
        if (t.size() != 3) throw std::runtime_error("boundary syntax: boundary <x> <y>");
        if ((t[1] != "p" && t[1] != "periodic") || (t[2] != "p" && t[2] != "periodic"))
            throw std::runtime_error("This solver only supports periodic (p) boundary.");
    } else if (cmd == "grid") {
        if (t.size() != 3) throw std::runtime_error("grid syntax: grid <Nx> <Ny>");
        c.active_nx = std::stoi(t[1]);
        c.active_ny = std::stoi(t[2]);
        if (c.active_nx <= 0 || c.active_ny <= 0) throw std::runtime_error("grid sizes must be positive");
        if (c.active_nx % 2 != 0 || c.active_ny % 2 != 0) throw std::runtime_error("grid must be even.");
        update_grid(s);
    } else if (cmd == "length") {
        if (t.size() != 3) throw std::runtime_error("length syntax: length <Lx> <Ly>");
        c.lx = std::stod(t[1]);
        c.ly = std::stod(t[2]);
        if (c.lx <= 0.0 || c.ly <= 0.0) throw std::runtime_error("domain lengths must be positive");
    } else if (cmd == "dealias") {
        if (t.size() != 2) throw std::runtime_error("dealias syntax: dealias <none|three_halves|3/2|two|2>");
        const std::string& r = t[1];
        if (r == "none" || r == "off") s.dealias = 0;
        else if (r == "three_halves" || r == "3/2") s.dealias = 1;
        else if (r == "two" || r == "2") s.dealias = 2;
        else throw std::runtime_error("unknown dealias rule: " + r);
        update_grid(s);
    } else if (cmd == "timestep") {
        if (t.size() != 2) throw std::runtime_error("timestep syntax: timestep <dt>");
        c.dt = std::stod(t[1]);
        if (c.dt <= 0.0) throw std::runtime_error("timestep must be positive");
    } else if (cmd == "time_evolution") {
        if (t.size() != 2) throw std::runtime_error("time_evolution syntax: time_evolution <type>");
        s.time_evolution = t[1];
    } else if (cmd == "model") {
        parse_model(s, t);
    } else if (cmd == "fix") {
        parse_fix(s, t);
    } else if (cmd == "set" || cmd == "thermo" || cmd == "restart") {
        // initial conditions / logging / restart: not part of the step
    } else if (cmd == "measure") {
        if (t.size() < 4) throw std::runtime_error("measure syntax: measure <ID> <type> <on|off> <args...>");
        s.commands_started = true;
    } else if (cmd == "run") {
        if (t.size() != 2) throw std::runtime_error("run syntax: run <steps>");
        if (std::stoi(t[1]) <= 0) throw std::runtime_error("run steps must be positive");
        s.commands_started = true;
    } else {
        throw std::runtime_error("Unknown command: " + cmd);
    }
}

void finish(ParseState& s) {
    shhd_config& c = s.cfg;
    const std::string& te = s.time_evolution;
    if (te == "euler/compressible") { c.integrator = SHHD_EULER; c.mode = SHHD_COMPRESSIBLE; }
    else if (te == "euler/incompressible") { c.integrator = SHHD_EULER; c.mode = SHHD_INCOMPRESSIBLE; }
    else if (te == "euler/quiescent") { c.integrator = SHHD_EULER; c.mode = SHHD_QUIESCENT; }
    else if (te == "srk3/compressible") { c.integrator = SHHD_SRK3; c.mode = SHHD_COMPRESSIBLE; }
    else if (te == "srk3/incompressible") { c.integrator = SHHD_SRK3; c.mode = SHHD_INCOMPRESSIBLE; }
    else if (te == "srk3/quiescent") { c.integrator = SHHD_SRK3; c.mode = SHHD_QUIESCENT; }
    else throw std::runtime_error("unknown time_evolution type: " + te);
    // validate_configuration (param_parser.cc:771-805)
    if (!s.has_transport) throw std::runtime_error("model transport must be specified");
    const bool quiet = is_quiescent(te);
    if (c.order_parameter_advection && c.num_order_parameters == 0)
        throw std::runtime_error("fix nonlinear order_parameter requires at least one order parameter.");
    if (quiet && c.momentum_advection) throw std::runtime_error("quiescent time evolution cannot use momentum nonlinear advection.");
    if (quiet && c.order_parameter_advection) throw std::runtime_error("quiescent time evolution cannot use order_parameter nonlinear advection.");
    for (int i = 0; i < c.n_sine_forces; ++i)
        if (quiet && c.sine_forces[i].target == 0) throw std::runtime_error("quiescent time evolution cannot use momentum force/sine.");
    if (quiet && c.n_gradient_forces > 0) throw std::runtime_error("quiescent time evolution cannot use force/gradient.");
}

}  // namespace

extern "C" {

int shhd_config_default(shhd_config* cfg) {
    if (!cfg) return SHHD_EINVAL;
    std::memset(cfg, 0, sizeof(*cfg));
    // src/simulationinfo.h:35-98
    cfg->active_nx = cfg->active_ny = 128;
    cfg->nx = cfg->ny = 128;
    cfg->lx = cfg->ly = 2.0 * 3.14159265358979323846;
    cfg->dt = 0.005;
    cfg->mode = SHHD_COMPRESSIBLE;
    cfg->integrator = SHHD_SRK3;
    cfg->noise_seed = 12345;
    cfg->kBT = 1.0;
    cfg->chi = 1.0;
    cfg->precision = SHHD_FP64;
    cfg->noise_source = SHHD_NOISE_PHILOX;
    cfg->batch = 1;
    return SHHD_OK;
}

}  // extern "C"

// the message is read back through shhd_last_error (engine.cu)
namespace shhd_internal {
void set_last_error(const std::string& msg);
}

extern "C" int shhd_config_from_script(const char* script_text, shhd_config* cfg) {
    if (!script_text || !cfg) {
        shhd_internal::set_last_error("null argument");
        return SHHD_EINVAL;
    }
    ParseState s;
    shhd_config_default(&s.cfg);
    try {
        std::istringstream in(script_text);
        std::string line;
        while (std::getline(in, line)) {
            const std::string clean = line.substr(0, line.find('#'));
            std::istringstream ls(clean);
            Tokens t;
            std::string w;
            while (ls >> w) t.push_back(w);
            execute(s, t);
        }
        finish(s);
    } catch (const std::exception& e) {
        shhd_internal::set_last_error(e.what());
        return SHHD_EINVAL;
    }
    *cfg = s.cfg;
    return SHHD_OK;
}
