// d3_cli: command-line D3 dispersion for structure files, on libd3.so.
//
// Drop-in for the reference's d3_cpp (LASP-D3 src/main.cpp): the same positional
// arguments and `--use-atm` switch, the same defaults (rc 60 bohr, CN and ATM cutoffs
// 40 bohr, zero damping, PBE, float I/O through the reference ABI) and the same report
// (cell, elapsed time, energy, per-atom forces, force sum, stress). Additions: extended
// XYZ input, cutoffs / damping / functional options, the FP64 path (--fp64), the
// precision form (--precision) and --parse-only (reads and prints the structures, no
// GPU).
//
//   d3_cli [--use-atm] [--rc B] [--rc-cn B] [--rc-atm B] [--damping zero|bj]
//          [--functional pbe|pbe0|b3lyp|blyp|bp86|revpbe] [--fp64] [--precision]
//          [--quiet] [--parse-only] file.arc|file.xyz|file.extxyz ...
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

#include "d3.h"

namespace {

const char *kSymbols[] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar",
    "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge", "As", "Se", "Br", "Kr",
    "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe",
    "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf",
    "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No", "Lr"};

int atomic_number(std::string s) {
    if (s.empty()) return -1;
    s[0] = (char)std::toupper((unsigned char)s[0]);
    for (size_t k = 1; k < s.size(); ++k) s[k] = (char)std::tolower((unsigned char)s[k]);
    for (int z = 0; z < (int)(sizeof(kSymbols) / sizeof(kSymbols[0])); ++z)
        if (s == kSymbols[z]) return z + 1;
    return -1;
}

struct Structure {
    std::vector<double> pos; // [n][3] Angstrom
    std::vector<uint16_t> Z;
    double cell[9] = {0};    // rows = lattice vectors, Angstrom
    bool has_cell = false;
};

std::vector<std::string> split(const std::string &line) {
    std::istringstream is(line);
    std::vector<std::string> t;
    std::string w;
    while (is >> w) t.push_back(w);
    return t;
}

// lengths (A) and angles (degrees) -> rows a, b, c with a along x and b in the xy plane
void cell_from_parameters(double a, double b, double c, double alpha, double beta, double gamma, double *h) {
    const double d2r = std::acos(-1.0) / 180.0;
    const double ca = std::cos(alpha * d2r), cb = std::cos(beta * d2r), cg = std::cos(gamma * d2r);
    const double sg = std::sin(gamma * d2r);
    const double cx = c * cb, cy = c * (ca - cb * cg) / sg;
    const double cz = std::sqrt(std::max(c * c - cx * cx - cy * cy, 0.0));
    const double v[9] = {a, 0.0, 0.0, b * cg, b * sg, 0.0, cx, cy, cz};
    std::memcpy(h, v, sizeof(v));
}

// .arc blocks: "Energy <n> <force> <energy> [sym]", "PBC a b c alpha beta gamma", and
// ten-token atom lines "symbol x y z ..."; other lines ("end") are skipped
bool read_arc(const std::string &path, std::vector<Structure> &out, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    Structure *cur = nullptr;
    while (std::getline(f, line)) {
        const auto t = split(line);
        if (t.empty()) continue;
        if (t[0] == "Energy" && (t.size() == 4 || t.size() == 5)) {
            out.emplace_back();
            cur = &out.back();
        } else if (t[0] == "PBC" && t.size() == 7 && cur) {
            cell_from_parameters(std::stod(t[1]), std::stod(t[2]), std::stod(t[3]), std::stod(t[4]), std::stod(t[5]),
                                 std::stod(t[6]), cur->cell);
            cur->has_cell = true;
        } else if (t.size() == 10 && cur) {
            const int z = atomic_number(t[0]);
            if (z < 1) {
                err = "unknown element " + t[0];
                return false;
            }
            cur->Z.push_back((uint16_t)z);
            for (int k = 1; k <= 3; ++k) cur->pos.push_back(std::stod(t[k]));
        }
    }
    return true;
}

// extended XYZ frames: count, comment with Lattice="...", "symbol x y z ..." lines
bool read_extxyz(const std::string &path, std::vector<Structure> &out, std::string &err) {
    std::ifstream f(path);
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    std::string line;
    const std::regex lat("Lattice\\s*=\\s*\"([^\"]+)\"");
    while (std::getline(f, line)) {
        const auto t = split(line);
        if (t.empty()) continue;
        const long n = std::stol(t[0]);
        std::string comment;
        if (!std::getline(f, comment)) break;
        std::smatch m;
        Structure s;
        if (!std::regex_search(comment, m, lat)) {
            err = path + ": frame without Lattice";
            return false;
        }
        const auto c = split(m[1].str());
        if (c.size() != 9) {
            err = path + ": Lattice needs 9 numbers";
            return false;
        }
        for (int k = 0; k < 9; ++k) s.cell[k] = std::stod(c[k]);
        s.has_cell = true;
        for (long a = 0; a < n; ++a) {
            if (!std::getline(f, line)) {
                err = path + ": truncated frame";
                return false;
            }
            const auto u = split(line);
            const int z = u.empty() ? -1 : atomic_number(u[0]);
            if (z < 1 || u.size() < 4) {
                err = path + ": bad atom line: " + line;
                return false;
            }
            s.Z.push_back((uint16_t)z);
            for (int k = 1; k <= 3; ++k) s.pos.push_back(std::stod(u[k]));
        }
        out.push_back(std::move(s));
    }
    return true;
}

bool ends_with(const std::string &s, const std::string &e) {
    return s.size() >= e.size() && s.compare(s.size() - e.size(), e.size(), e) == 0;
}

void usage() {
    std::cout << "Usage: d3_cli [options] file.arc|file.xyz|file.extxyz ...\n"
                 "Options:\n"
                 "  -h, --help          Display this help message\n"
                 "  --use-atm           Include the ATM three-body term\n"
                 "  --rc B              two-body cutoff in bohr (default 60)\n"
                 "  --rc-cn B           coordination-number cutoff in bohr (default 40)\n"
                 "  --rc-atm B          ATM cutoff in bohr (default 40)\n"
                 "  --damping zero|bj   damping function (default zero)\n"
                 "  --functional NAME   pbe, pbe0, b3lyp, blyp, bp86, revpbe (default pbe)\n"
                 "  --fp64              double-precision input/output path\n"
                 "  --precision         FP32 pair/triplet arithmetic (precision form)\n"
                 "  --quiet             print only the energy of each structure\n"
                 "  --parse-only        read and print the structures, no evaluation\n";
}

} // namespace

int main(int argc, char **argv) {
    std::vector<std::string> files;
    bool use_atm = false, fp64 = false, precision = false, quiet = false, parse_only = false;
    double rc = 60.0, rc_cn = 40.0, rc_atm = 40.0;
    int damping = ZERO_DAMPING, functional = PBE;
    const std::map<std::string, int> funcs = {{"pbe", PBE},   {"pbe0", PBE0}, {"b3lyp", B3LYP},
                                              {"blyp", BLYP}, {"bp86", BP86}, {"revpbe", REVPBE}};
    if (argc < 2) {
        std::cerr << "No input file provided. Use -h or --help for usage." << std::endl;
        return EXIT_FAILURE;
    }
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&](const char *name) -> std::string {
            if (i + 1 >= argc) {
                std::cerr << name << " needs a value" << std::endl;
                std::exit(EXIT_FAILURE);
            }
            return argv[++i];
        };
        if (a == "-h" || a == "--help") {
            usage();
            return 0;
        } else if (a == "--use-atm") {
            use_atm = true;
        } else if (a == "--rc") {
            rc = std::stod(value("--rc"));
        } else if (a == "--rc-cn") {
            rc_cn = std::stod(value("--rc-cn"));
        } else if (a == "--rc-atm") {
            rc_atm = std::stod(value("--rc-atm"));
        } else if (a == "--damping") {
            const std::string d = value("--damping");
            if (d == "zero")
                damping = ZERO_DAMPING;
            else if (d == "bj")
                damping = BJ_DAMPING;
            else {
                std::cerr << "unknown damping " << d << std::endl;
                return EXIT_FAILURE;
            }
        } else if (a == "--functional") {
            const std::string f = value("--functional");
            if (!funcs.count(f)) {
                std::cerr << "unknown functional " << f << std::endl;
                return EXIT_FAILURE;
            }
            functional = funcs.at(f);
        } else if (a == "--fp64") {
            fp64 = true;
        } else if (a == "--precision") {
            precision = true;
        } else if (a == "--quiet") {
            quiet = true;
        } else if (a == "--parse-only") {
            parse_only = true;
        } else if (std::ifstream(a).good()) {
            files.push_back(a);
        } else {
            std::cerr << "Unknown argument or file does not exist: " << a << std::endl;
            return EXIT_FAILURE;
        }
    }
    for (const auto &file : files) {
        std::vector<Structure> structures;
        std::string err;
        const bool ok = (ends_with(file, ".xyz") || ends_with(file, ".extxyz")) ? read_extxyz(file, structures, err)
                                                                                : read_arc(file, structures, err);
        if (!ok || structures.empty()) {
            std::cerr << "Error parsing file: " << file << (err.empty() ? "" : ": " + err) << std::endl;
            return EXIT_FAILURE;
        }
        if (!quiet) std::cout << "Parsed " << structures.size() << " structures from file: " << file << std::endl;
        for (const auto &s : structures) {
            const uint64_t n = s.Z.size();
            if (!s.has_cell) {
                std::cerr << "structure without a cell in " << file << std::endl;
                return EXIT_FAILURE;
            }
            if (!quiet || parse_only) {
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        std::cout << "Cell[" << i << "][" << j << "]: " << std::setprecision(10) << s.cell[3 * i + j]
                                  << std::endl;
            }
            if (parse_only) {
                std::cout << "Atoms: " << n << std::endl;
                continue;
            }
            if (!quiet) std::cout << "Computing dispersion energy for " << n << " atoms..." << std::endl;
            std::vector<uint16_t> el(s.Z);
            d3_handle_t *h = nullptr;
            if (fp64)
                h = d3_init_handle_ex(el.data(), n, n, rc, rc_cn, use_atm ? rc_atm : 0.0, damping, functional,
                                      D3_TABLE_5REF);
            else if (use_atm)
                h = init_d3_handle_with_atm(el.data(), n, n, (real_t)rc, (real_t)rc_cn, (real_t)rc_atm,
                                            (damping_type_t)damping, (functional_t)functional);
            else
                h = init_d3_handle(el.data(), n, n, (real_t)rc, (real_t)rc_cn, (damping_type_t)damping,
                                   (functional_t)functional);
            if (!h) {
                std::cerr << "Failed to initialize D3 handle: " << d3_last_error() << std::endl;
                return EXIT_FAILURE;
            }
            if (precision) d3_set_option(h, D3_OPT_PRECISION, 1);
            std::vector<double> F(3 * n), S(9);
            double energy = 0.0;
            uint16_t st = 0;
            const auto t0 = std::chrono::high_resolution_clock::now();
            if (fp64) {
                d3_set_cell_f64(h, s.cell);
                d3_set_atoms_f64(h, s.pos.data(), el.data(), n);
                st = d3_compute_f64(h, &energy, F.data(), S.data());
            } else {
                std::vector<float> posf(s.pos.begin(), s.pos.end()), Ff(3 * n), Sf(9);
                float cellf[3][3];
                for (int k = 0; k < 9; ++k) cellf[k / 3][k % 3] = (float)s.cell[k];
                float e = 0.0f;
                set_atoms(h, posf.data(), el.data(), n);
                set_cell(h, cellf);
                clear_d3_handle(h);
                st = compute_dispersion_energy_from_handle_status(h, &e, Ff.data(), Sf.data());
                energy = e;
                for (size_t k = 0; k < F.size(); ++k) F[k] = Ff[k];
                for (int k = 0; k < 9; ++k) S[k] = Sf[k];
            }
            const double elapsed =
                std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
            free_d3_handle(h);
            if (st != 0) {
                std::cerr << "evaluation status " << st << ": " << d3_last_error() << std::endl;
                return EXIT_FAILURE;
            }
            if (quiet) {
                std::cout << std::setprecision(12) << energy << std::endl;
                continue;
            }
            std::cout << "Elapsed time: " << elapsed << " seconds" << std::endl;
            std::cout << std::fixed << std::setprecision(20) << "Energy: " << energy << " eV" << std::endl;
            double fsum[3] = {0, 0, 0};
            for (uint64_t i = 0; i < n; ++i) {
                for (int k = 0; k < 3; ++k) fsum[k] += F[3 * i + k];
                std::cout << "Force[" << i << "]: " << F[3 * i] << " " << F[3 * i + 1] << " " << F[3 * i + 2]
                          << std::endl;
            }
            std::cout << "Force sum: " << fsum[0] << " " << fsum[1] << " " << fsum[2] << std::endl;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    std::cout << "Stress[" << i << "][" << j << "]: " << S[3 * i + j] << std::endl;
            std::cout.unsetf(std::ios::fixed);
        }
    }
    return EXIT_SUCCESS;
}
