// vd_run -- C++ host driver of the library, the counterpart of the
// reference's executable main loop (Source/main.cpp: read the inputs file,
// construct Vidyut, Evolve until max_step or stop_time).  It drives one case
// library through the C ABI of include/vidyut_b200.h only:
//
//   vd_run <inputs> [key=value ...] [--check] [--dump <file>]
//
// The inputs file and the command-line overrides use the reference's
// ParmParse syntax ("name = value ...", '#' comments).  Keys:
//   max_step, stop_time                    loop limits (as the reference);
//   prob.*                                 handed to vd_init_domain (the
//                                          case's amrex_probinit);
//   amr.plot_int, amr.plot_file            raw state dumps every plot_int
//                                          steps (<plot_file><step>.bin);
//   everything else (vidyut.*, geometry.*, amr.n_cell)  vd_config_set.
// The dimension follows the number of amr.n_cell entries, as the reference's
// DIM build switch fixes it.  --check parses and validates the inputs and
// prints the resolved configuration without touching a GPU.  --dump writes
// the final state (all components, FP64, x fastest) to <file>.
//
// A raw dump is "VDST" then int32 dim, nx, ny, nz, ncomp, int32 step, FP64
// time, then the components one after another.
#include <vidyut_b200.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

std::string trim(const std::string& s)
{
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// One "name = value" per line; later definitions win, as in ParmParse.
void parse_line(const std::string& raw, std::vector<std::pair<std::string, std::string>>& kv)
{
    std::string line = raw.substr(0, raw.find('#'));
    const size_t eq = line.find('=');
    if (eq == std::string::npos) return;
    const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
    if (!k.empty()) kv.emplace_back(k, v);
}

int count_words(const std::string& v)
{
    std::istringstream is(v);
    std::string w;
    int n = 0;
    while (is >> w) ++n;
    return n;
}

const char* status_name(int s)
{
    switch (s)
    {
    case VD_OK: return "VD_OK";
    case VD_ERR_INVALID_ARG: return "VD_ERR_INVALID_ARG";
    case VD_ERR_CUDA: return "VD_ERR_CUDA";
    case VD_ERR_NOT_CONVERGED: return "VD_ERR_NOT_CONVERGED";
    case VD_ERR_UNSUPPORTED: return "VD_ERR_UNSUPPORTED";
    case VD_ERR_OOM: return "VD_ERR_OOM";
    case VD_ERR_NONFINITE: return "VD_ERR_NONFINITE";
    }
    return "unknown";
}

int fail(void* ctx, const char* what, int st)
{
    char msg[512] = {0};
    vd_last_error(ctx, msg, sizeof(msg));
    std::fprintf(stderr, "vd_run: %s failed: %s %s\n", what, status_name(st), msg);
    return 1;
}

bool dump(void* ctx, const vd_config& cfg, const vd_case_info_t& info, const std::string& path,
          double time, int step)
{
    const long long n = (long long)cfg.n_cell[0] * cfg.n_cell[1] * (cfg.dim == 3 ? cfg.n_cell[2] : 1);
    std::vector<double> s((size_t)n * info.nvar);
    if (vd_get_state(ctx, 0, info.nvar, s.data(), 0) != VD_OK) return false;
    std::ofstream f(path, std::ios::binary);
    const int32_t hdr[6] = {cfg.dim, cfg.n_cell[0], cfg.n_cell[1], cfg.dim == 3 ? cfg.n_cell[2] : 1,
                            info.nvar, step};
    f.write("VDST", 4);
    f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
    f.write(reinterpret_cast<const char*>(&time), sizeof(time));
    f.write(reinterpret_cast<const char*>(s.data()), (std::streamsize)(s.size() * sizeof(double)));
    return bool(f);
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: %s <inputs> [key=value ...] [--check] [--dump <file>]\n", argv[0]);
        return 2;
    }
    std::vector<std::pair<std::string, std::string>> kv;
    {
        std::ifstream in(argv[1]);
        if (!in)
        {
            std::fprintf(stderr, "vd_run: cannot read %s\n", argv[1]);
            return 2;
        }
        std::string line;
        while (std::getline(in, line)) parse_line(line, kv);
    }
    bool check = false;
    std::string dump_path;
    for (int a = 2; a < argc; ++a)
    {
        if (!std::strcmp(argv[a], "--check")) check = true;
        else if (!std::strcmp(argv[a], "--dump") && a + 1 < argc) dump_path = argv[++a];
        else parse_line(argv[a], kv);
    }
    std::map<std::string, std::string> last;
    for (auto& p : kv) last[p.first] = p.second;

    vd_config cfg;
    vd_config_init(&cfg);
    if (last.count("amr.n_cell")) cfg.dim = count_words(last["amr.n_cell"]) == 2 ? 2 : 3;
    int max_step = 1 << 30, plot_int = -1;
    double stop_time = 1e300;
    std::string plot_file = "plt", prob;
    for (auto& p : kv)
    {
        const std::string& k = p.first;
        const std::string& v = p.second;
        if (k == "max_step") max_step = std::atoi(v.c_str());
        else if (k == "stop_time") stop_time = std::atof(v.c_str());
        else if (k == "amr.plot_int") plot_int = std::atoi(v.c_str());
        else if (k == "amr.plot_file") plot_file = v;
        else if (k.rfind("prob.", 0) == 0) prob += k + " = " + v + "\n";
        else
        {
            const int st = vd_config_set(&cfg, k.c_str(), v.c_str());
            if (st == VD_ERR_INVALID_ARG)
                std::fprintf(stderr, "vd_run: ignoring unknown or malformed key %s = %s\n",
                             k.c_str(), v.c_str());
            else if (st != VD_OK)
                std::fprintf(stderr, "vd_run: key %s not supported (%s)\n", k.c_str(),
                             status_name(st));
        }
    }
    vd_case_info_t info;
    vd_case_info(&info);
    std::printf("case %s: %d species, %d components; dim %d, n_cell %d %d %d, dt %.6g, "
                "hyp_order %d, weno_scheme %d, correctors %d, max_step %d, stop_time %.6g\n",
                info.case_name, info.num_species, info.nvar, cfg.dim, cfg.n_cell[0],
                cfg.n_cell[1], cfg.n_cell[2], cfg.dt, cfg.hyp_order, cfg.weno_scheme,
                cfg.num_timestep_correctors, max_step, stop_time);
    if (check) return 0;

    void* ctx = nullptr;
    int st = vd_create(&cfg, &ctx);
    if (st != VD_OK) return fail(nullptr, "vd_create", st);
    st = vd_init_domain(ctx, prob.c_str());
    if (st != VD_OK) return fail(ctx, "vd_init_domain", st);
    double time = 0.0;
    int step = 0;
    while (step < max_step && time < stop_time)
    {
        vd_step_stats ss;
        st = vd_step(ctx, 1, &ss);
        if (st != VD_OK && st != VD_ERR_NOT_CONVERGED) return fail(ctx, "vd_step", st);
        vd_get_time(ctx, &time, &step);
        std::printf("step %d time %.9g dt %.6g poisson V-cycles %d species V-cycles %d gpu %.3f ms%s\n",
                    step, time, ss.dt, ss.poisson_iterations, ss.species_iterations, ss.gpu_ms,
                    st == VD_ERR_NOT_CONVERGED ? " (a solve hit linsolve_maxiter)" : "");
        if (plot_int > 0 && step % plot_int == 0)
        {
            char name[512];
            std::snprintf(name, sizeof(name), "%s%05d.bin", plot_file.c_str(), step);
            if (!dump(ctx, cfg, info, name, time, step)) return fail(ctx, "state dump", VD_ERR_CUDA);
        }
    }
    long long bad = 0;
    vd_check_state(ctx, &bad);
    if (!dump_path.empty() && !dump(ctx, cfg, info, dump_path, time, step))
        return fail(ctx, "state dump", VD_ERR_CUDA);
    vd_destroy(ctx);
    if (bad)
    {
        std::fprintf(stderr, "vd_run: %lld non-finite values in the state\n", bad);
        return 1;
    }
    return 0;
}
