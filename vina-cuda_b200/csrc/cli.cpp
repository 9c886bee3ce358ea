// vdock command-line front end: the reference's --config CLI and PDBQT output
// (main.cpp:569-1020 options and config file, 89-102 write_all_output,
// 159-170 REMARK VINA RESULT, 460-489 result table) over the C ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/vdock.h"

namespace fs = std::filesystem;

static void die(const std::string& m) {
    std::fprintf(stderr, "\n\nError: %s\n", m.c_str());
    std::exit(1);
}
static void check(vd_status s, const char* what) {
    if (s != VD_OK) die(std::string(what) + ": " + vd_last_error());
}
static std::string slurp(const std::string& path) {
    std::ifstream f(path);
    if (!f) die("could not open \"" + path + "\" for reading.");
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}
static std::string trim(std::string s) {
    while (!s.empty() && std::isspace((unsigned char)s.back())) s.pop_back();
    size_t i = 0;
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    return s.substr(i);
}

static const char* kUsage =
    "Input:\n  --receptor arg  --ligand arg  --ligand_directory arg  --output_directory arg\n"
    "  --thread arg (chains per ligand)  --search_depth arg  --rilc_bfgs arg (default 1)\n"
    "Search space (required):\n  --center_x/y/z arg  --size_x/y/z arg\n"
    "Output (optional):\n  --out arg  --log arg\n"
    "Advanced:\n  --weight_gauss1 --weight_gauss2 --weight_repulsion --weight_hydrophobic\n"
    "  --weight_hydrogen --weight_rot\n"
    "Misc:\n  --seed arg  --num_modes arg (9)  --energy_range arg (3)  --device arg (0)\n"
    "  --batch arg (ligands per batched launch, 64)\n"
    "Configuration file:\n  --config arg   (key = value lines with the options above)\n";

int main(int argc, char** argv) {
    std::map<std::string, std::string> opt;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--help") { std::printf("%s", kUsage); return 0; }
        if (a == "--version") { std::printf("vdock (B200) AutoDock-Vina-compatible docking\n"); return 0; }
        if (a.rfind("--", 0) != 0 || i + 1 >= argc) {
            std::fprintf(stderr, "Command line parse error: %s\n\nCorrect usage:\n%s", a.c_str(), kUsage);
            return 1;
        }
        opt[a.substr(2)] = argv[++i];
    }
    if (opt.count("config")) {  // command-line values win over the file (boost program_options order)
        std::istringstream cf(slurp(opt["config"]));
        std::string line;
        while (std::getline(cf, line)) {
            const size_t h = line.find('#');
            if (h != std::string::npos) line = line.substr(0, h);
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
            if (!k.empty() && !opt.count(k)) opt[k] = v;
        }
    }
    auto num = [&](const char* k, double d) { return opt.count(k) ? std::atof(opt[k].c_str()) : d; };
    if (!opt.count("receptor")) { std::fprintf(stderr, "Missing receptor.\n\nCorrect usage:\n%s", kUsage); return 1; }
    if (!opt.count("ligand") && !opt.count("ligand_directory")) { std::fprintf(stderr, "Missing ligand\n"); return 1; }
    if (opt.count("ligand") && opt.count("ligand_directory")) {
        std::fprintf(stderr, "Can not define ligand and ligand_directory at the same time\n");
        return 1;
    }
    for (const char* k : {"center_x", "center_y", "center_z", "size_x", "size_y", "size_z"})
        if (!opt.count(k)) { std::fprintf(stderr, "Missing search space option --%s\n\nCorrect usage:\n%s", k, kUsage); return 1; }
    const double center[3] = {num("center_x", 0), num("center_y", 0), num("center_z", 0)};
    const double size[3] = {num("size_x", 0), num("size_y", 0), num("size_z", 0)};
    if (size[0] <= 0 || size[1] <= 0 || size[2] <= 0) die("Search space dimensions should be positive");
    const int thread = int(num("thread", 8192));
    if (thread < 1000) die("thread must be at least 1000");
    const int search_depth = int(num("search_depth", 0));
    if (opt.count("search_depth") && search_depth < 1) die("search_depth must be 1 or greater");
    if (int(num("rilc_bfgs", 1)) != 1)
        std::fprintf(stderr, "WARNING: only the RILC-BFGS local search is implemented; using it\n");
    const double w_rot = num("weight_rot", 0.05846);
    const double weights[6] = {num("weight_gauss1", -0.035579), num("weight_gauss2", -0.005156),
                               num("weight_repulsion", 0.840245), num("weight_hydrophobic", -0.035069),
                               num("weight_hydrogen", -0.587439), 5 * w_rot / 0.1 - 1};

    std::vector<std::string> ligs, outs;
    if (opt.count("ligand")) {
        ligs.push_back(opt["ligand"]);
        std::string o = opt.count("out") ? opt["out"] : opt["ligand"];
        if (!opt.count("out")) {
            if (o.size() >= 6 && o.substr(o.size() - 6) == ".pdbqt") o.resize(o.size() - 6);
            o += "_out.pdbqt";
        }
        outs.push_back(o);
    } else {
        const std::string dir = opt["ligand_directory"];
        const std::string odir = opt.count("output_directory") ? opt["output_directory"] : dir + "_out";
        fs::create_directories(odir);
        std::vector<fs::path> files;
        for (auto& e : fs::directory_iterator(dir))
            if (e.path().extension() == ".pdbqt") files.push_back(e.path());
        std::sort(files.begin(), files.end());
        for (auto& f : files) {
            ligs.push_back(f.string());
            outs.push_back((fs::path(odir) / (f.stem().string() + "_out.pdbqt")).string());
        }
        std::printf("Output will be in the directory %s\n", odir.c_str());
    }

    vd_ctx* ctx = nullptr;
    check(vd_create(&ctx, int(num("device", 0))), "vd_create");
    check(vd_set_scoring(ctx, weights), "vd_set_scoring");
    vd_pdbqt* rh = nullptr;
    int32_t nr = 0;
    const double* rxyz = nullptr;
    const int32_t* rxs = nullptr;
    check(vd_pdbqt_receptor(slurp(opt["receptor"]).c_str(), &rh, &nr, &rxyz, &rxs), "receptor");
    check(vd_set_receptor(ctx, nr, rxyz, rxs), "vd_set_receptor");
    check(vd_set_box(ctx, center, size), "vd_set_box");

    std::vector<vd_pdbqt*> handles;
    std::vector<vd_ligand_desc> descs;
    std::vector<int32_t> ids;
    std::vector<std::string> kept_out;
    bool need[VD_XS_TYPES] = {};
    for (size_t i = 0; i < ligs.size(); ++i) {
        vd_pdbqt* h = nullptr;
        vd_ligand_desc d;
        if (vd_pdbqt_ligand(slurp(ligs[i]).c_str(), &h, &d) != VD_OK) {
            std::fprintf(stderr, "\nParse error in file \"%s\": %s\n", ligs[i].c_str(), vd_last_error());
            continue;
        }
        int32_t id = -1;
        if (vd_add_ligand(ctx, &d, &id) != VD_OK) {
            std::fprintf(stderr, "skipping %s: %s\n", ligs[i].c_str(), vd_last_error());
            vd_pdbqt_free(h);
            continue;
        }
        for (int a = 0; a < d.n_atoms; ++a)
            if (d.xs[a] >= 0) need[d.xs[a]] = true;
        handles.push_back(h);
        descs.push_back(d);
        ids.push_back(id);
        kept_out.push_back(outs[i]);
    }
    if (ids.empty()) die("No valid ligands");
    std::vector<int32_t> types;
    for (int t = 0; t < VD_XS_TYPES; ++t)
        if (need[t]) types.push_back(t);
    check(vd_build_grids(ctx, types.data(), int32_t(types.size())), "vd_build_grids");

    vd_search_params sp{};
    sp.seed = opt.count("seed") ? uint32_t(std::strtoul(opt["seed"].c_str(), nullptr, 10)) : 12345u;
    sp.n_chains = thread;
    sp.search_depth = search_depth;
    sp.max_bfgs_steps = 0;
    sp.num_modes = int(num("num_modes", 9));
    sp.energy_range = num("energy_range", 3.0);
    sp.hunt_cap[0] = sp.hunt_cap[1] = sp.hunt_cap[2] = 10;
    sp.temperature = 1.2;
    sp.amplitude = 2.0;
    sp.min_rmsd = 1.0;
    sp.refine = 1;
    std::vector<vd_dock_result> res(ids.size());
    const int batch = std::max(1, int(num("batch", 64)));
    for (size_t b = 0; b < ids.size(); b += batch) {
        const int n = int(std::min(ids.size() - b, size_t(batch)));
        if (n == 1) check(vd_dock_plain(ctx, ids[b], &sp, &res[b]), "vd_dock_plain");
        else check(vd_dock_batched(ctx, &ids[b], n, &sp, &res[b]), "vd_dock_batched");
    }
    FILE* log = opt.count("log") ? std::fopen(opt["log"].c_str(), "w") : nullptr;
    for (size_t i = 0; i < ids.size(); ++i) {
        const vd_dock_result& r = res[i];
        std::string table = "mode |   affinity | dist from best mode\n     | (kcal/mol) | rmsd l.b.| rmsd u.b.\n"
                            "-----+------------+----------+----------\n";
        std::ofstream f(kept_out[i]);
        if (!f) die("could not open \"" + kept_out[i] + "\" for writing.");
        std::vector<double> xyz(3 * size_t(descs[i].n_atoms));
        for (int m = 0; m < r.n_modes; ++m) {
            char line[128];
            std::snprintf(line, sizeof line, "%4d    %9.1f  %9.3f  %9.3f\n", m + 1, r.energy[m], r.rmsd_lb[m], r.rmsd_ub[m]);
            table += line;
            check(vd_conf_to_coords(&descs[i], r.pose[m], xyz.data()), "vd_conf_to_coords");
            int64_t len = 0;
            check(vd_pdbqt_write_model(handles[i], xyz.data(), nullptr, 0, &len), "write");
            std::string buf(size_t(len) + 1, '\0');
            check(vd_pdbqt_write_model(handles[i], xyz.data(), &buf[0], len + 1, &len), "write");
            char remark[128];
            std::snprintf(remark, sizeof remark, "REMARK VINA RESULT: %9.1f  %9.3f  %9.3f\n", r.energy[m], r.rmsd_lb[m],
                          r.rmsd_ub[m]);
            f << "MODEL " << m + 1 << "\n" << remark << buf.c_str() << "ENDMDL\n";
        }
        if (r.n_modes < 1)
            table += "WARNING: Could not find any conformations completely within the search space.\n";
        std::printf("%s\n%s", ligs.size() > 1 ? kept_out[i].c_str() : "", table.c_str());
        if (log) std::fprintf(log, "%s", table.c_str());
    }
    if (log) std::fclose(log);
    for (auto* h : handles) vd_pdbqt_free(h);
    vd_pdbqt_free(rh);
    vd_destroy(ctx);
    return 0;
}
