// gpulouvain_main.cpp -- the `gpulouvain -f file.mtx -g min-gain [-v]` CLI.
//
// Same flags and stdout as the reference's main (gpulouvain.cu:6-46,
// utils.cu:161-186): line 1 the final modularity ("%f"), line 2
// "algorithmTime totalTime" in milliseconds, then with -v the map of
// printOriginalToCommunity (modularity_optimisation.cu:403-418).  Timing
// scopes follow the reference: totalTime adds the device set-up (allocation,
// host->device copy, M) to the algorithm time (level loop + final modularity);
// reading the file is not timed.
//
// Not in the reference: -d N selects the CUDA device, and -c keeps a binary
// CSR cache beside the file (<file>.lvcsr, lv_write_csr_stamped): the cache
// records the text file's size and modification time (nanoseconds) and is
// read instead of the text only while both still match the file.  Without
// -c the parsed entries are copied to the device and the CSR is built there
// (lv_csr_from_entries_device; the same CSR as the host build), timed as the
// reference times its host->device copy.  --mode learned runs the learned
// active-set sweeps with a predictor file (--model FILE; default: the
// packaged active_set_lfr.json beside the bin/ directory) and the settings
// stored in it; the partition is then no longer the plain rule's.
#include <getopt.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/louvain_b200.h"

// The CSR of `file`, through the cache <file>.lvcsr when use_cache is set.
static int read_graph(const char *file, bool use_cache, int32_t *V, int64_t *E, int32_t **rowptr, int32_t **col,
                      float **w) {
    if (!use_cache) return lv_read_mtx(file, V, E, rowptr, col, w, nullptr);
    const std::string cache = std::string(file) + ".lvcsr";
    struct stat sf;
    const bool have_stat = stat(file, &sf) == 0;
    const int64_t size = have_stat ? (int64_t)sf.st_size : 0;
    const int64_t mtime_ns = have_stat ? (int64_t)sf.st_mtim.tv_sec * 1000000000LL + sf.st_mtim.tv_nsec : 0;
    int64_t c_size = 0, c_mtime = 0;
    if (have_stat && lv_read_csr_stamp(cache.c_str(), &c_size, &c_mtime) == LV_OK && c_size == size &&
        c_mtime == mtime_ns && lv_read_csr(cache.c_str(), V, E, rowptr, col, w, nullptr) == LV_OK)
        return LV_OK;
    float m_ref = 0;
    const int rc = lv_read_mtx(file, V, E, rowptr, col, w, &m_ref);
    if (rc == LV_OK && have_stat &&
        lv_write_csr_stamped(cache.c_str(), *V, *E, *rowptr, *col, *w, m_ref, size, mtime_ns) != LV_OK)
        std::fprintf(stderr, "gpulouvain: could not write the cache %s\n", cache.c_str());
    return rc;
}

static void usage() {
    std::printf("Usage: ./gpulouvain -f mtx-matrix-file -g min-gain [-v]\n");
    std::exit(1);
}

// The packaged predictor: ../active_set_lfr.json relative to this binary.
static std::string packaged_model() {
    char exe[4096];
    const ssize_t n = readlink("/proc/self/exe", exe, sizeof exe - 1);
    if (n <= 0) return "active_set_lfr.json";
    exe[n] = 0;
    std::string dir(exe);
    const size_t slash = dir.rfind('/');
    dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
    return dir + "/../active_set_lfr.json";
}

int main(int argc, char *argv[]) {
    const char *file = nullptr;
    float min_gain = 0;
    bool have_f = false, have_g = false, verbose = false, use_cache = false;
    int device = 0;
    bool learned = false;
    std::string model_path;
    static const struct option long_opts[] = {{"mode", required_argument, nullptr, 'm'},
                                              {"model", required_argument, nullptr, 'M'},
                                              {nullptr, 0, nullptr, 0}};
    int opt;
    while ((opt = getopt_long(argc, argv, "f:g:vd:c", long_opts, nullptr)) != -1) {
        switch (opt) {
        case 'g': have_g = true; min_gain = std::strtof(optarg, nullptr); break;
        case 'v': verbose = true; break;
        case 'f': have_f = true; file = optarg; break;
        case 'd': device = std::atoi(optarg); break;
        case 'c': use_cache = true; break;
        case 'm':
            if (std::strcmp(optarg, "learned") == 0) learned = true;
            else if (std::strcmp(optarg, "plain") != 0) usage();
            break;
        case 'M': model_path = optarg; break;
        default: usage();
        }
    }
    if (!have_f || !have_g) usage();

    lv_opts opts;
    lv_default_opts(&opts);
    opts.device = device;
    std::vector<uint16_t> model(LV_ACTIVE_MODEL_SIZE);
    int32_t n_params = 0;
    float logit_thr = 0;
    if (learned) {
        if (model_path.empty()) model_path = packaged_model();
        const int mrc = lv_read_active_model(model_path.c_str(), model.data(), (int32_t)model.size(), &n_params,
                                             &logit_thr, &opts);
        if (mrc != LV_OK) {
            std::fprintf(stderr, "gpulouvain: cannot read the predictor %s: %s\n", model_path.c_str(),
                         lv_status_string(mrc));
            return EXIT_FAILURE;
        }
    }

    int32_t V = 0;
    int64_t E = 0;
    int32_t *rowptr = nullptr, *col = nullptr;   // host CSR (-c) or device CSR
    float *w = nullptr;
    int32_t *ea = nullptr, *eb = nullptr;           // parsed entries (no -c)
    float *ew = nullptr;
    int64_t nnz = 0;
    int rc = use_cache ? read_graph(file, true, &V, &E, &rowptr, &col, &w)
                       : lv_read_mtx_entries(file, &V, &nnz, &ea, &eb, &ew);
    if (rc != LV_OK) {
        std::fprintf(stderr, "gpulouvain: cannot read %s: %s\n", file, lv_status_string(rc));
        return EXIT_FAILURE;
    }
    using clk = std::chrono::steady_clock;
    lv_handle *h = nullptr;
    auto t0 = clk::now();
    if (use_cache) {
        rc = lv_create(rowptr, col, w, V, E, &opts, &h);
    } else {
        rc = lv_csr_from_entries_device(device, V, nnz, ea, eb, ew, &E, &rowptr, &col, &w);
        if (rc == LV_OK) rc = lv_create_device(rowptr, col, w, V, E, &opts, &h);
    }
    if (rc == LV_OK && learned) rc = lv_set_active_model(h, model.data(), n_params, logit_thr);
    auto t1 = clk::now();
    if (rc != LV_OK) {
        std::fprintf(stderr, "gpulouvain: %s\n", lv_status_string(rc));
        return EXIT_FAILURE;
    }
    double q = 0;
    auto t2 = clk::now();
    rc = lv_run(h, min_gain, &q);
    auto t3 = clk::now();
    if (rc != LV_OK) {
        std::fprintf(stderr, "gpulouvain: %s: %s\n", lv_status_string(rc), lv_last_error(h));
        lv_destroy(h);
        return EXIT_FAILURE;
    }
    const double memory_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    const double algo_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
    std::printf("%f\n", q);
    std::printf("%f %f\n", algo_ms, algo_ms + memory_ms);
    if (verbose) {
        int32_t *o2c = (int32_t *)std::malloc(sizeof(int32_t) * (size_t)(V > 0 ? V : 1));
        int32_t nc = 0;
        rc = lv_get_original_to_community(h, o2c, &nc);
        if (rc == LV_OK) {
            std::fflush(stdout);
            rc = lv_print_communities(nullptr, o2c, V, nc);
        }
        std::free(o2c);
    }
    lv_destroy(h);
    if (use_cache) {
        lv_free_host(rowptr);
        lv_free_host(col);
        lv_free_host(w);
    } else {
        lv_free_device(rowptr);
        lv_free_device(col);
        lv_free_device(w);
        lv_free_host(ea);
        lv_free_host(eb);
        lv_free_host(ew);
    }
    return rc == LV_OK ? 0 : EXIT_FAILURE;
}
