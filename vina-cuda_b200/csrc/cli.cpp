// vdock command-line front end: the reference's --config CLI and PDBQT output
// (main.cpp:569-1020 options and config file, 89-102 write_all_output,
// 159-170 REMARK VINA RESULT, 460-489 result table) over the C ABI.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
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
// Ligand files parsed on worker threads ahead of the docking loop, at most
// `ahead` files past the consumer (bounded memory); results are consumed in
// file order so ligand ids -- and with them the random streams -- do not
// depend on parse timing.
class ParsePool {
  public:
    struct Slot {
        vd_pdbqt* h = nullptr;
        vd_ligand_desc d{};
        bool ok = false;
        std::string err;
    };
    ParsePool(const std::vector<std::string>& files, size_t ahead, unsigned threads)
        : files_(files), slots_(files.size()), ready_(files.size(), 0), ahead_(std::max<size_t>(1, ahead)) {
        for (unsigned t = 0; t < std::max(1u, threads); ++t) th_.emplace_back([this] { work(); });
    }
    ~ParsePool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_space_.notify_all();
        for (auto& t : th_) t.join();
        for (size_t i = 0; i < slots_.size(); ++i)  // parsed but never consumed
            if (ready_[i] && !taken_[i] && slots_[i].h) vd_pdbqt_free(slots_[i].h);
    }
    // Blocks until file i is parsed; the caller owns the slot's handle.
    Slot take(size_t i) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_ready_.wait(lk, [&] { return ready_[i] != 0; });
        taken_[i] = 1;
        consumed_ = i + 1;
        cv_space_.notify_all();
        return slots_[i];
    }

  private:
    void work() {
        for (;;) {
            size_t i;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_space_.wait(lk, [&] { return stop_ || next_ >= files_.size() || next_ < consumed_ + ahead_; });
                if (stop_ || next_ >= files_.size()) return;
                i = next_++;
            }
            Slot s;
            std::ifstream f(files_[i]);
            if (!f) {
                s.err = "could not open \"" + files_[i] + "\" for reading";
            } else {
                std::stringstream ss;
                ss << f.rdbuf();
                if (vd_pdbqt_ligand(ss.str().c_str(), &s.h, &s.d) == VD_OK) s.ok = true;
                else s.err = vd_last_error();
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                slots_[i] = s;
                ready_[i] = 1;
            }
            cv_ready_.notify_all();
        }
    }
    std::vector<std::string> files_;
    std::vector<Slot> slots_;
    std::vector<char> ready_, taken_ = std::vector<char>(files_.size(), 0);
    size_t ahead_, next_ = 0, consumed_ = 0;
    bool stop_ = false;
    std::mutex mu_;
    std::condition_variable cv_ready_, cv_space_;
    std::vector<std::thread> th_;
};

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
    "  --visited_history arg (0; 1 = QuickVina2-CUDA's visited history, with --rilc_bfgs 1)\n"
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
    const int rilc_bfgs = int(num("rilc_bfgs", 1));  // main.cpp:663: 1 = RILC-BFGS, 0 = dense BFGS
    if (rilc_bfgs != 0 && rilc_bfgs != 1) die("rilc_bfgs must be 0 or 1");
    const int visited = int(num("visited_history", 0));  // QuickVina2-CUDA's search policy
    if (visited != 0 && visited != 1) die("visited_history must be 0 or 1");
    if (visited && !rilc_bfgs) die("visited_history needs --rilc_bfgs 1");
    const double w_rot = num("weight_rot", 0.05846);
    const double weights[6] = {num("weight_gauss1", -0.035579), num("weight_gauss2", -0.005156),
                               num("weight_repulsion", 0.840245), num("weight_hydrophobic", -0.035069),
                               num("weight_hydrogen", -0.587439), 5 * w_rot / 0.1 - 1};

    std::vector<std::string> ligs, outs;
    const bool directory = opt.count("ligand_directory") != 0;
    if (!directory) {
        ligs.push_back(opt["ligand"]);
        std::string o = opt.count("out") ? opt["out"] : opt["ligand"];
        if (!opt.count("out")) {
            if (o.size() >= 6 && o.substr(o.size() - 6) == ".pdbqt") o.resize(o.size() - 6);
            o += "_out.pdbqt";
        }
        outs.push_back(o);
    } else {  // every file of the directory (main.cpp:897-945), in name order; unparsable ones are skipped
        const std::string dir = opt["ligand_directory"];
        const std::string odir = opt.count("output_directory") ? opt["output_directory"] : dir + "_out";
        fs::create_directories(odir);
        std::vector<fs::path> files;
        for (auto& e : fs::directory_iterator(dir))
            if (e.is_regular_file()) files.push_back(e.path());
        std::sort(files.begin(), files.end());
        for (auto& f : files) {
            ligs.push_back(f.string());
            std::string stem = f.filename().string();
            const size_t dot = stem.find(".pdbqt");
            if (dot != std::string::npos) stem.resize(dot);
            outs.push_back((fs::path(odir) / (stem + "_out.pdbqt")).string());
        }
        std::printf("Output will be in the directory %s\n", odir.c_str());
    }
    const auto t_start = std::chrono::steady_clock::now();

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

    const int batch = std::max(1, int(num("batch", 64)));
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    ParsePool pool(ligs, size_t(4) * batch, std::min(hw, 16u));
    // maps: a single ligand's types; for a directory all 17 (as the reference
    // builds them, main_procedure_cu.cpp:167-175), so docking starts while
    // later files are still being parsed
    std::vector<int32_t> types;
    ParsePool::Slot first;
    if (!directory) {
        first = pool.take(0);
        if (!first.ok) {
            std::fprintf(stderr, "\nParse error in file \"%s\": %s\n", ligs[0].c_str(), first.err.c_str());
            return 1;
        }
        bool need[VD_XS_TYPES] = {};
        for (int a = 0; a < first.d.n_atoms; ++a)
            if (first.d.xs[a] >= 0) need[first.d.xs[a]] = true;
        for (int t = 0; t < VD_XS_TYPES; ++t)
            if (need[t]) types.push_back(t);
    } else {
        for (int t = 0; t < VD_XS_TYPES; ++t) types.push_back(t);
    }
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
    sp.dense_bfgs = rilc_bfgs == 0;
    sp.visited_history = visited;
    FILE* log = opt.count("log") ? std::fopen(opt["log"].c_str(), "w") : nullptr;

    struct Item {
        size_t file;
        ParsePool::Slot s;
        int32_t id;
    };
    std::vector<Item> pending;
    size_t n_docked = 0;
    auto run_batch = [&]() {
        // the batch's ligands are packed together on host threads; if one is
        // rejected, they are added one by one and the rejected ones skipped
        std::vector<vd_ligand_desc> descs;
        for (auto& it : pending) descs.push_back(it.s.d);
        std::vector<int32_t> ids(pending.size());
        if (vd_add_ligands(ctx, descs.data(), int32_t(descs.size()), ids.data()) != VD_OK) {
            std::vector<Item> kept;
            ids.clear();
            for (auto& it : pending) {
                if (vd_add_ligand(ctx, &it.s.d, &it.id) != VD_OK) {
                    std::fprintf(stderr, "skipping %s: %s\n", ligs[it.file].c_str(), vd_last_error());
                    vd_pdbqt_free(it.s.h);
                    continue;
                }
                kept.push_back(it);
                ids.push_back(it.id);
            }
            pending.swap(kept);
            if (pending.empty()) return;
        } else {
            for (size_t k = 0; k < pending.size(); ++k) pending[k].id = ids[k];
        }
        std::vector<vd_dock_result> res(ids.size());
        if (ids.size() == 1) check(vd_dock_plain(ctx, ids[0], &sp, &res[0]), "vd_dock_plain");
        else check(vd_dock_batched(ctx, ids.data(), int32_t(ids.size()), &sp, res.data()), "vd_dock_batched");
        for (size_t k = 0; k < pending.size(); ++k) {
            const Item& it = pending[k];
            const vd_dock_result& r = res[k];
            const std::string& out = outs[it.file];
            std::string table = "mode |   affinity | dist from best mode\n     | (kcal/mol) | rmsd l.b.| rmsd u.b.\n"
                                "-----+------------+----------+----------\n";
            std::ofstream f(out);
            if (!f) die("could not open \"" + out + "\" for writing.");
            std::vector<double> xyz(3 * size_t(it.s.d.n_atoms));
            for (int m = 0; m < r.n_modes; ++m) {
                char line[128];
                std::snprintf(line, sizeof line, "%4d    %9.1f  %9.3f  %9.3f\n", m + 1, r.energy[m], r.rmsd_lb[m],
                              r.rmsd_ub[m]);
                table += line;
                check(vd_conf_to_coords(&it.s.d, r.pose[m], xyz.data()), "vd_conf_to_coords");
                int64_t len = 0;
                check(vd_pdbqt_write_model(it.s.h, xyz.data(), nullptr, 0, &len), "write");
                std::string buf(size_t(len) + 1, '\0');
                check(vd_pdbqt_write_model(it.s.h, xyz.data(), &buf[0], len + 1, &len), "write");
                char remark[128];
                std::snprintf(remark, sizeof remark, "REMARK VINA RESULT: %9.1f  %9.3f  %9.3f\n", r.energy[m],
                              r.rmsd_lb[m], r.rmsd_ub[m]);
                f << "MODEL " << m + 1 << "\n" << remark << buf.c_str() << "ENDMDL\n";
            }
            if (r.n_modes < 1)
                table += "WARNING: Could not find any conformations completely within the search space.\n";
            std::printf("%s\n%s", directory ? out.c_str() : "", table.c_str());
            if (log) std::fprintf(log, "%s", table.c_str());
            vd_pdbqt_free(it.s.h);
        }
        n_docked += pending.size();
        pending.clear();
    };
    for (size_t i = 0; i < ligs.size(); ++i) {
        ParsePool::Slot s = (i == 0 && !directory) ? first : pool.take(i);
        if (!s.ok) {
            std::fprintf(stderr, "\nParse error in file \"%s\": %s\n", ligs[i].c_str(), s.err.c_str());
            continue;
        }
        pending.push_back({i, s, -1});  // added with the rest of its batch
        if (int(pending.size()) == batch) run_batch();
    }
    if (!pending.empty()) run_batch();
    if (n_docked == 0) die(directory ? "No valid ligands in the input directory" : "No valid ligands");
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    if (directory) std::printf("Docked %zu ligands in %.2f s\n", n_docked, secs);
    if (log) std::fclose(log);
    vd_pdbqt_free(rh);
    vd_destroy(ctx);
    return 0;
}
