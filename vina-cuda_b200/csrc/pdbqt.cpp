// PDBQT ingestion and output for the drop-in CLI.
//
//   grammar and atom columns     lib/parse_pdbqt.cpp:101-118, 262-401
//   atom order / rigid bodies    parse_pdbqt.cpp:342-401 (postprocess_branch)
//   covalent bonds               lib/model.cpp:644-700 (assign_bonds, bead order)
//   XS typing                    model.cpp:771-798
//   intra pairs                  model.cpp:836-900 (bonded_to depth 3)
//   N_tors                       lib/terms.cpp:97-128
//   output lines                 model.cpp:1063-1116 (coordinates patched into
//                                the input lines, %8.3f at columns 31/39/47)
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <functional>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace {

const char* kAdNames[20] = {"C", "A", "N", "O", "P", "S", "H", "F", "I", "NA",
                            "OA", "SA", "HD", "Mg", "Mn", "Zn", "Ca", "Fe", "Cl", "Br"};
const double kAdCov[20] = {0.77, 0.77, 0.75, 0.73, 1.06, 1.02, 0.37, 0.71, 1.33, 0.75,
                           0.73, 1.02, 0.37, 1.30, 1.39, 1.31, 1.74, 1.25, 0.99, 1.14};
const int kAdEl[20] = {1, 1, 2, 3, 5, 4, 0, 6, 9, 2, 3, 4, 0, 10, 10, 10, 10, 10, 7, 8};
const char* kMetals[9] = {"Cu", "Fe", "Na", "K", "Hg", "Co", "U", "Cd", "Ni"};
const double kMaxCov = 1.74;
enum { FIXED = 0, ROTOR = 1, VARIABLE = 2 };

struct PAtom {
    int number = 0;
    int ad = 20;      // AD type, 20 = none (metal)
    bool metal = false;
    double xyz[3] = {0, 0, 0};
    int line = 0;     // index into the stored lines
    int el() const { return ad < 20 ? kAdEl[ad] : (metal ? 10 : 11); }
    double cov() const { return ad < 20 ? kAdCov[ad] : 1.75; }
    bool hydrogen() const { return ad == 6 || ad == 12; }
    bool hetero() const { return (ad != 0 && ad != 1 && ad != 6 && ad != 12 && ad < 20) || metal; }
};

struct ParseError {
    std::string msg;
};

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
    while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
    return s.substr(a, b - a);
}

bool starts(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

PAtom parse_atom(const std::string& s, int line_no) {
    PAtom a;
    auto field = [&](size_t i, size_t j) {  // 1-based inclusive columns
        if (j > s.size()) throw ParseError{"line " + std::to_string(line_no) + ": the line is too short"};
        return trim(s.substr(i - 1, j - i + 1));
    };
    try {
        a.number = std::stoi(field(7, 11));
        for (int k = 0; k < 3; ++k) a.xyz[k] = std::stod(field(31 + 8 * k, 38 + 8 * k));
    } catch (const std::exception&) {
        throw ParseError{"line " + std::to_string(line_no) + ": ATOM syntax incorrect"};
    }
    std::string name = s.size() >= 78 ? trim(s.substr(77)) : "";
    if (name == "Se") name = "S";
    for (int i = 0; i < 20; ++i)
        if (name == kAdNames[i]) { a.ad = i; break; }
    for (const char* m : kMetals)
        if (name == m) a.metal = true;
    if (a.ad == 20 && !a.metal)
        throw ParseError{"line " + std::to_string(line_no) + ": \"" + name + "\" is not a valid AutoDock type"};
    return a;
}

bool is_atom_line(const std::string& s) { return starts(s, "ATOM  ") || starts(s, "HETATM"); }
bool is_ignorable(const std::string& s) { return s.empty() || starts(s, "WARNING") || starts(s, "REMARK"); }

// Parse-tree node: atoms of one ROOT/BRANCH block and their sub-branches.
struct Block {
    struct Node {
        PAtom a;
        std::vector<std::unique_ptr<Block>> kids;
    };
    std::vector<Node> atoms;
    int immobile = -1;
    int axis_begin = -1, axis_end = -1;
    bool essentially_empty() const {
        for (size_t i = 0; i < atoms.size(); ++i) {
            if (immobile >= 0 && immobile != int(i)) return false;
            if (!atoms[i].kids.empty()) return false;
        }
        return true;
    }
};

struct Lines {
    std::vector<std::string> v;
    size_t pos = 0;
    bool next(std::string& s) {
        if (pos >= v.size()) return false;
        s = v[pos++];
        if (!s.empty() && s.back() == '\r') s.pop_back();
        return true;
    }
};

void parse_branch(Lines& in, Block& b, int from, int to);

void branch_aux(Lines& in, Block& b, const std::string& s) {
    int first = 0, second = 0;
    if (std::sscanf(s.c_str() + 6, "%d %d", &first, &second) != 2)
        throw ParseError{"line " + std::to_string(in.pos) + ": Syntax error"};
    for (auto& nd : b.atoms)
        if (nd.a.number == first) {
            nd.kids.emplace_back(new Block());
            parse_branch(in, *nd.kids.back(), first, second);
            return;
        }
    throw ParseError{"line " + std::to_string(in.pos) + ": No atom number " + std::to_string(first) + " in this branch"};
}

void parse_branch(Lines& in, Block& b, int from, int to) {
    std::string s;
    while (in.next(s)) {
        if (is_ignorable(s)) continue;
        if (starts(s, "BRANCH")) branch_aux(in, b, s);
        else if (starts(s, "ENDBRANCH")) {
            int f = 0, t = 0;
            std::sscanf(s.c_str() + 9, "%d %d", &f, &t);
            if (f != from || t != to) throw ParseError{"line " + std::to_string(in.pos) + ": Inconsistent branch numbers"};
            if (b.immobile < 0)
                throw ParseError{"line " + std::to_string(in.pos) + ": Atom " + std::to_string(to) +
                                 " has not been found in this branch"};
            return;
        } else if (is_atom_line(s)) {
            PAtom a = parse_atom(s, int(in.pos));
            a.line = int(in.pos) - 1;
            if (a.number == to) b.immobile = int(b.atoms.size());
            b.atoms.push_back({a, {}});
        } else {
            throw ParseError{"line " + std::to_string(in.pos) + ": Unknown or inappropriate tag"};
        }
    }
    throw ParseError{"unexpected end of file inside a BRANCH"};
}

}  // namespace

struct vd_pdbqt {
    std::vector<std::string> lines;
    std::vector<PAtom> atoms;            // model order
    std::vector<int32_t> line_of_atom;
    std::vector<double> xyz;
    std::vector<int32_t> xs, el, atom_node, node_parent, node_origin, node_axis, pairs;
    double num_tors = 0;
    int torsdof = 0;
};

namespace {

double d2(const double* a, const double* b) {
    return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
}

// Bonds by distance among atoms whose mutual mobility is not VARIABLE.
// mob(i,j) answers the mobility; bead order fixes the bond order.
template <class Mob>
std::vector<std::vector<std::pair<int, bool>>> perceive_bonds(const std::vector<PAtom>& A, Mob mob) {
    const int n = int(A.size());
    std::vector<std::pair<const double*, std::vector<int>>> beads;
    for (int i = 0; i < n; ++i) {
        bool put = false;
        for (auto& b : beads)
            if (d2(A[i].xyz, b.first) < 15.0 * 15.0) { b.second.push_back(i); put = true; break; }
        if (!put) beads.emplace_back(A[i].xyz, std::vector<int>(1, i));
    }
    std::vector<std::vector<std::pair<int, bool>>> bonds(n);
    for (int i = 0; i < n; ++i) {
        const double ci = A[i].cov();
        const double bead_cut = (15 + 1.1 * (ci + kMaxCov)) * (15 + 1.1 * (ci + kMaxCov));
        std::vector<int> rel;
        for (auto& b : beads) {
            if (d2(b.first, A[i].xyz) > bead_cut) continue;
            for (int j : b.second)
                if (j != i && mob(i, j) != VARIABLE &&
                    d2(A[i].xyz, A[j].xyz) < (1.1 * (ci + kMaxCov)) * (1.1 * (ci + kMaxCov)))
                    rel.push_back(j);
        }
        for (int j : rel) {
            if (j <= i) continue;
            const double r2 = d2(A[i].xyz, A[j].xyz);
            const double bl = ci + A[j].cov();
            if (!(r2 < (1.1 * bl) * (1.1 * bl))) continue;
            bool between = false;
            for (int c : rel) {
                if (c == i || c == j) continue;
                if (mob(i, c) != VARIABLE && mob(j, c) != VARIABLE && d2(A[i].xyz, A[c].xyz) < r2 &&
                    d2(A[j].xyz, A[c].xyz) < r2) {
                    between = true;
                    break;
                }
            }
            if (between) continue;
            const bool rot = mob(i, j) == ROTOR;
            bonds[i].push_back({j, rot});
            bonds[j].push_back({i, rot});
        }
    }
    return bonds;
}

int xs_of(const PAtom& a, bool bonded_hetero, bool bonded_hd) {
    const int el = a.el();
    const bool acceptor = a.ad == 9 || a.ad == 10;
    const bool donor = el == 10 || bonded_hd;
    switch (el) {
        case 0: return -1;
        case 1: return bonded_hetero ? 1 : 0;
        case 2: return (acceptor && donor) ? 5 : (acceptor ? 4 : (donor ? 3 : 2));
        case 3: return (acceptor && donor) ? 9 : (acceptor ? 8 : (donor ? 7 : 6));
        case 4: return 10;
        case 5: return 11;
        case 6: return 12;
        case 7: return 13;
        case 8: return 14;
        case 9: return 15;
        case 10: return 16;
        default: return -1;
    }
}

void build_ligand(vd_pdbqt& P, Block& root) {
    std::vector<std::array<int, 4>> writes;  // kind, a, b, c : mobility writes in order
    int n_nodes = 0;
    std::function<void(Block&, int)> process = [&](Block& b, int k) {
        const int begin = int(P.atoms.size());
        auto insert = [&](Block::Node& nd) {
            for (auto& kid : nd.kids) kid->axis_begin = int(P.atoms.size());
            P.atoms.push_back(nd.a);
            P.atom_node.push_back(k);
        };
        for (size_t i = 0; i < b.atoms.size(); ++i) {
            if (!(b.immobile >= 0 && int(i) == b.immobile)) insert(b.atoms[i]);
            for (auto& kid : b.atoms[i].kids)
                if (!kid->atoms.empty()) {
                    kid->axis_end = int(P.atoms.size());
                    insert(kid->atoms[kid->immobile]);
                }
        }
        const int end = int(P.atoms.size());
        if (b.axis_begin >= 0) writes.push_back({0, b.axis_begin, begin, end});
        if (b.axis_end >= 0) writes.push_back({0, b.axis_end, begin, end});
        if (b.axis_begin >= 0 && b.axis_end >= 0) writes.push_back({1, b.axis_begin, b.axis_end, 0});
        writes.push_back({2, begin, end, 0});
        for (auto& nd : b.atoms)
            for (auto& kid : nd.kids)
                if (!kid->essentially_empty()) {
                    const int kk = n_nodes++;
                    P.node_parent.push_back(k);
                    P.node_origin.push_back(kid->axis_end);
                    P.node_axis.push_back(kid->axis_begin);
                    process(*kid, kk);
                }
    };
    n_nodes = 1;
    P.node_parent.push_back(-1);
    P.node_origin.push_back(0);
    P.node_axis.push_back(-1);
    process(root, 0);
    const int n = int(P.atoms.size());
    std::vector<uint8_t> mob(size_t(n) * n, VARIABLE);
    for (auto& w : writes) {
        if (w[0] == 0) {
            for (int i = w[2]; i < w[3]; ++i) mob[size_t(w[1]) * n + i] = mob[size_t(i) * n + w[1]] = FIXED;
        } else if (w[0] == 1) {
            mob[size_t(w[1]) * n + w[2]] = mob[size_t(w[2]) * n + w[1]] = ROTOR;
        } else {
            for (int i = w[1]; i < w[2]; ++i)
                for (int j = w[1]; j < w[2]; ++j) mob[size_t(i) * n + j] = FIXED;
        }
    }
    for (int i = 0; i < n; ++i) mob[size_t(i) * n + i] = FIXED;
    auto m = [&](int i, int j) { return int(mob[size_t(i) * n + j]); };
    auto bonds = perceive_bonds(P.atoms, m);
    P.xs.resize(n);
    P.el.resize(n);
    for (int i = 0; i < n; ++i) {
        bool het = false, hd = false;
        for (auto& b : bonds[i]) {
            het |= P.atoms[b.first].hetero();
            hd |= P.atoms[b.first].ad == 12;
        }
        P.xs[i] = xs_of(P.atoms[i], het, hd);
        P.el[i] = P.atoms[i].el();
    }
    for (int i = 0; i < n; ++i) {
        std::vector<int> near;  // bonded_to(i, 3): DFS with a visited list
        std::function<void(int, int)> dfs = [&](int a, int depth) {
            if (std::find(near.begin(), near.end(), a) != near.end()) return;
            near.push_back(a);
            if (depth > 0)
                for (auto& b : bonds[a]) dfs(b.first, depth - 1);
        };
        dfs(i, 3);
        for (int j = i + 1; j < n; ++j)
            if (m(i, j) == VARIABLE && std::find(near.begin(), near.end(), j) == near.end() && P.xs[i] >= 0 &&
                P.xs[j] >= 0) {
                P.pairs.push_back(i);
                P.pairs.push_back(j);
            }
    }
    auto heavy_nb = [&](int k) {
        int c = 0;
        for (auto& b : bonds[k]) c += !P.atoms[b.first].hydrogen();
        return c;
    };
    double nt = 0;
    for (int i = 0; i < n; ++i) {
        if (P.el[i] == 0) continue;
        int ar = 0;
        for (auto& b : bonds[i])
            if (b.second && !P.atoms[b.first].hydrogen() && heavy_nb(b.first) > 1) ++ar;
        nt += 0.5 * ar;
    }
    P.num_tors = nt;
    P.xyz.resize(3 * size_t(n));
    P.line_of_atom.resize(n);
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) P.xyz[3 * i + k] = P.atoms[i].xyz[k];
        P.line_of_atom[i] = P.atoms[i].line;
    }
}

}  // namespace

using namespace vd;

extern "C" {

vd_status vd_pdbqt_ligand(const char* text, vd_pdbqt** out, vd_ligand_desc* desc) {
    VD_CHECK(text && out && desc, VD_ERR_ARG, "vd_pdbqt_ligand: NULL argument");
    std::unique_ptr<vd_pdbqt> P(new vd_pdbqt());
    try {
        std::istringstream ss(text);
        std::string s;
        while (std::getline(ss, s)) P->lines.push_back(s);
        Lines in{P->lines, 0};
        Block root;
        bool in_root = false, have_tors = false;
        while (in.next(s)) {  // parse_pdbqt_root
            if (is_ignorable(s)) continue;
            if (starts(s, "ROOT")) { in_root = true; break; }
            throw ParseError{"line " + std::to_string(in.pos) + ": Unknown or inappropriate tag"};
        }
        if (!in_root) throw ParseError{"no ROOT record"};
        while (in.next(s)) {
            if (is_ignorable(s)) continue;
            if (is_atom_line(s)) {
                PAtom a = parse_atom(s, int(in.pos));
                a.line = int(in.pos) - 1;
                root.atoms.push_back({a, {}});
            } else if (starts(s, "ENDROOT")) break;
            else throw ParseError{"line " + std::to_string(in.pos) + ": Unknown or inappropriate tag"};
        }
        while (in.next(s)) {
            if (is_ignorable(s)) continue;
            if (starts(s, "BRANCH")) branch_aux(in, root, s);
            else if (starts(s, "TORSDOF")) {
                if (have_tors) throw ParseError{"line " + std::to_string(in.pos) + ": TORSDOF can occur only once"};
                P->torsdof = std::atoi(s.c_str() + 7);
                have_tors = true;
            } else throw ParseError{"line " + std::to_string(in.pos) + ": Unknown or inappropriate tag"};
        }
        if (root.atoms.empty()) throw ParseError{"No atoms in the ligand"};
        if (!have_tors) throw ParseError{"Missing TORSDOF"};
        build_ligand(*P, root);
    } catch (const ParseError& e) {
        set_error("PDBQT parse error: " + e.msg);
        return VD_ERR_PARSE;
    }
    desc->n_atoms = int32_t(P->atoms.size());
    desc->n_nodes = int32_t(P->node_parent.size());
    desc->n_pairs = int32_t(P->pairs.size() / 2);
    desc->xyz = P->xyz.data();
    desc->xs = P->xs.data();
    desc->el = P->el.data();
    desc->atom_node = P->atom_node.data();
    desc->node_parent = P->node_parent.data();
    desc->node_origin_atom = P->node_origin.data();
    desc->node_axis_atom = P->node_axis.data();
    desc->pairs = P->pairs.data();
    desc->num_tors = P->num_tors;
    *out = P.release();
    return VD_OK;
}

vd_status vd_pdbqt_receptor(const char* text, vd_pdbqt** out, int32_t* n_atoms, const double** xyz,
                            const int32_t** xs) {
    VD_CHECK(text && out && n_atoms && xyz && xs, VD_ERR_ARG, "vd_pdbqt_receptor: NULL argument");
    std::unique_ptr<vd_pdbqt> P(new vd_pdbqt());
    try {
        std::istringstream ss(text);
        std::string s;
        int no = 0;
        while (std::getline(ss, s)) {
            ++no;
            if (!s.empty() && s.back() == '\r') s.pop_back();
            if (s.empty() || starts(s, "TER") || starts(s, "WARNING") || starts(s, "REMARK")) continue;
            if (is_atom_line(s)) P->atoms.push_back(parse_atom(s, no));
            else if (starts(s, "MODEL")) throw ParseError{"line " + std::to_string(no) + ": Unexpected multi-MODEL input"};
            else throw ParseError{"line " + std::to_string(no) + ": Unknown or inappropriate tag"};
        }
    } catch (const ParseError& e) {
        set_error("PDBQT parse error: " + e.msg);
        return VD_ERR_PARSE;
    }
    // receptor atoms are mutually FIXED; bonds via a 3 A cell hash
    const int n = int(P->atoms.size());
    const double cell = 3.0;
    auto key = [&](const double* p, int dx, int dy, int dz) {
        long long x = (long long)std::floor(p[0] / cell) + dx, y = (long long)std::floor(p[1] / cell) + dy,
                  z = (long long)std::floor(p[2] / cell) + dz;
        return (x * 73856093LL) ^ (y * 19349663LL) ^ (z * 83492791LL);
    };
    std::unordered_map<long long, std::vector<int>> grid;
    for (int i = 0; i < n; ++i) grid[key(P->atoms[i].xyz, 0, 0, 0)].push_back(i);
    std::vector<char> het(n, 0), hd(n, 0);
    for (int i = 0; i < n; ++i) {
        const PAtom& a = P->atoms[i];
        const double reach = 1.1 * (a.cov() + kMaxCov);
        std::vector<int> rel;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = grid.find(key(a.xyz, dx, dy, dz));
                    if (it == grid.end()) continue;
                    for (int j : it->second)
                        if (j != i && d2(a.xyz, P->atoms[j].xyz) < reach * reach) rel.push_back(j);
                }
        std::sort(rel.begin(), rel.end());
        rel.erase(std::unique(rel.begin(), rel.end()), rel.end());
        for (int j : rel) {
            if (j <= i) continue;
            const double r2 = d2(a.xyz, P->atoms[j].xyz);
            const double bl = a.cov() + P->atoms[j].cov();
            if (!(r2 < (1.1 * bl) * (1.1 * bl))) continue;
            bool between = false;
            for (int c : rel)
                if (c != j && d2(a.xyz, P->atoms[c].xyz) < r2 && d2(P->atoms[j].xyz, P->atoms[c].xyz) < r2) {
                    between = true;
                    break;
                }
            if (between) continue;
            het[i] |= P->atoms[j].hetero();
            het[j] |= a.hetero();
            hd[i] |= P->atoms[j].ad == 12;
            hd[j] |= a.ad == 12;
        }
    }
    P->xyz.resize(3 * size_t(n));
    P->xs.resize(n);
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) P->xyz[3 * i + k] = P->atoms[i].xyz[k];
        P->xs[i] = xs_of(P->atoms[i], het[i], hd[i]);
    }
    *n_atoms = n;
    *xyz = P->xyz.data();
    *xs = P->xs.data();
    *out = P.release();
    return VD_OK;
}

vd_status vd_pdbqt_write_model(vd_pdbqt* P, const double* xyz_all, char* buf, int64_t size, int64_t* written) {
    VD_CHECK(P && xyz_all && written, VD_ERR_ARG, "vd_pdbqt_write_model: NULL argument");
    std::vector<int> atom_of_line(P->lines.size(), -1);
    for (size_t i = 0; i < P->line_of_atom.size(); ++i) atom_of_line[P->line_of_atom[i]] = int(i);
    std::string out;
    for (size_t l = 0; l < P->lines.size(); ++l) {
        std::string s = P->lines[l];
        if (!s.empty() && s.back() == '\r') s.pop_back();
        const int a = atom_of_line[l];
        if (a >= 0) {
            VD_CHECK(s.size() >= 54, VD_ERR_PARSE, "atom line too short to write coordinates");
            for (int k = 0; k < 3; ++k) {
                char f[32];
                std::snprintf(f, sizeof f, "%8.3f", xyz_all[3 * a + k]);
                VD_CHECK(std::strlen(f) == 8, VD_ERR_ARG, "coordinate does not fit %8.3f");
                s.replace(30 + 8 * k, 8, f);
            }
        }
        out += s;
        out += '\n';
    }
    *written = int64_t(out.size());
    if (buf) {
        VD_CHECK(size >= int64_t(out.size()) + 1, VD_ERR_ARG, "vd_pdbqt_write_model: buffer too small");
        std::memcpy(buf, out.c_str(), out.size() + 1);
    }
    return VD_OK;
}

vd_status vd_pdbqt_free(vd_pdbqt* P) {
    delete P;
    return VD_OK;
}

// tree.h:395-400 set_conf in double, all atoms (hydrogens included).
vd_status vd_conf_to_coords(const vd_ligand_desc* d, const float* pose, double* out) {
    VD_CHECK(d && pose && out, VD_ERR_ARG, "vd_conf_to_coords: NULL argument");
    const int nn = d->n_nodes, na = d->n_atoms;
    std::vector<double> q(4 * nn), o(3 * nn), R(9 * nn);
    auto qmat = [](const double* q, double* m) {
        const double a = q[0], b = q[1], c = q[2], e = q[3];
        m[0] = a * a + b * b - c * c - e * e; m[3] = 2 * (-a * e + b * c); m[6] = 2 * (a * c + b * e);
        m[1] = 2 * (a * e + b * c); m[4] = a * a - b * b + c * c - e * e; m[7] = 2 * (-a * b + c * e);
        m[2] = 2 * (-a * c + b * e); m[5] = 2 * (a * b + c * e); m[8] = a * a - b * b - c * c + e * e;
    };
    auto X = [&](int i, int k) { return d->xyz[3 * size_t(i) + k]; };
    for (int k = 0; k < nn; ++k) {
        if (k == 0) {
            for (int j = 0; j < 3; ++j) o[j] = pose[j];
            for (int j = 0; j < 4; ++j) q[j] = pose[3 + j];
        } else {
            const int p = d->node_parent[k];
            const int oa = d->node_origin_atom[k], pa = d->node_origin_atom[p], ax = d->node_axis_atom[k];
            double rel[3], axis[3], nrm = 0;
            for (int j = 0; j < 3; ++j) {
                rel[j] = X(oa, j) - X(pa, j);
                axis[j] = X(oa, j) - X(ax, j);
                nrm += axis[j] * axis[j];
            }
            nrm = std::sqrt(nrm);
            double al[3];
            for (int j = 0; j < 3; ++j) {
                axis[j] /= nrm;
                o[3 * k + j] = o[3 * p + j] + R[9 * p + j] * rel[0] + R[9 * p + 3 + j] * rel[1] + R[9 * p + 6 + j] * rel[2];
            }
            for (int j = 0; j < 3; ++j)
                al[j] = R[9 * p + j] * axis[0] + R[9 * p + 3 + j] * axis[1] + R[9 * p + 6 + j] * axis[2];
            const double th = 0.5 * pose[7 + k - 1], s = std::sin(th), c = std::cos(th);
            const double A[4] = {c, s * al[0], s * al[1], s * al[2]};
            const double* B = &q[4 * p];
            double* Q = &q[4 * k];
            Q[0] = A[0] * B[0] - A[1] * B[1] - A[2] * B[2] - A[3] * B[3];
            Q[1] = A[0] * B[1] + A[1] * B[0] + A[2] * B[3] - A[3] * B[2];
            Q[2] = A[0] * B[2] - A[1] * B[3] + A[2] * B[0] + A[3] * B[1];
            Q[3] = A[0] * B[3] + A[1] * B[2] - A[2] * B[1] + A[3] * B[0];
        }
        double* Q = &q[4 * k];
        const double inv = 1.0 / std::sqrt(Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]);
        for (int j = 0; j < 4; ++j) Q[j] *= inv;
        qmat(Q, &R[9 * k]);
    }
    for (int i = 0; i < na; ++i) {
        const int k = d->atom_node[i], oa = d->node_origin_atom[k];
        double l[3];
        for (int j = 0; j < 3; ++j) l[j] = X(i, j) - X(oa, j);
        for (int j = 0; j < 3; ++j)
            out[3 * i + j] = o[3 * k + j] + R[9 * k + j] * l[0] + R[9 * k + 3 + j] * l[1] + R[9 * k + 6 + j] * l[2];
    }
    return VD_OK;
}

}  // extern "C"
