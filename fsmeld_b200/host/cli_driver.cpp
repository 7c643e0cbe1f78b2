// Drop-ins for the reference's three entry points (include/funcs.h:64-72):
// read TARGET.bin / QUERY.txt, run the query on the GPU through the C ABI,
// and print what the reference prints.
//
//   fsmeld_search_file  <- FSMELD                (src/fsmeld.cpp:570-1074)
//   fsmeld_cutoff_file  <- FSMELD_find_threshold (src/fsmeld.cpp:185-569)
//   fsmeld_exact_file   <- FSMELD_exact          (src/fsmeld.cpp:1075-1344)
//
// Output formats follow the reference line for line: iostream's default
// six significant digits are printf("%g") and setprecision(17) is "%.17g";
// the experiment CSV follows src/search_result.cpp:39-101.  Differences by
// design: timings are this implementation's; the cutoff command's progress
// lines show the device's search bound (the reference shows its running
// heap threshold) and its pruning counters are the device's.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <string>
#include <vector>

#include <unistd.h>

#include "../../include/fsmeld_cuda.h"

namespace {

int metric_of(const char* tag) {
    if (!tag) return 0;
    if (!strcmp(tag, "dtw")) return FSMELD_DTW;
    if (!strcmp(tag, "edr")) return FSMELD_EDR;
    if (!strcmp(tag, "erp")) return FSMELD_ERP;
    if (!strcmp(tag, "lcss")) return FSMELD_LCSS;
    if (!strcmp(tag, "msm")) return FSMELD_MSM;
    return 0;
}

int device_index() {
    const char* d = std::getenv("FSMELD_DEVICE");
    return d ? std::atoi(d) : 0;
}

// FSMELD_NORMALIZATION=raw selects the raw mode (fsmeld_set_normalization);
// the reference's command line always runs z-score (src/main.cpp:89)
bool raw_mode() {
    const char* v = std::getenv("FSMELD_NORMALIZATION");
    return v != nullptr && std::string(v) == "raw";
}

bool quiet_matches() {  // src/fsmeld.cpp:998-1001
    const char* v = std::getenv("FSMELD_QUIET_MATCHES");
    return v != nullptr && std::string(v) != "0" && std::string(v) != "false";
}

// fscanf("%lf") loop of src/fsmeld.cpp:622-632
bool read_query(const char* path, int m, std::vector<double>* q) {
    FILE* f = fopen(path, "r");
    if (!f) return false;
    q->clear();
    double d;
    while ((int)q->size() < m && fscanf(f, "%lf", &d) == 1) q->push_back(d);
    fclose(f);
    return (int)q->size() == m;
}

std::string csv_escape(const std::string& v) {  // src/search_result.cpp:13-22
    if (v.find_first_of(",\"\r\n") == std::string::npos) return v;
    std::string e = "\"";
    for (char ch : v) {
        if (ch == '"') e += '"';
        e += ch;
    }
    return e + "\"";
}

std::string g17(double x) {
    char b[64];
    snprintf(b, sizeof(b), "%.17g", x);
    return b;
}

std::string timestamp_now() {
    const std::time_t now = std::time(nullptr);
    std::tm lt{};
    localtime_r(&now, &lt);
    char b[32];
    std::strftime(b, sizeof(b), "%Y-%m-%dT%H:%M:%S", &lt);
    return b;
}

std::string dataset_name(const char* path) {  // src/search_result.cpp:71-76
    if (!path || !*path) return "unknown";
    std::filesystem::path p(path);
    const std::filesystem::path parent = p.parent_path();
    return parent.empty() ? p.stem().string() : parent.filename().string();
}

struct Row {
    std::string dataset, metric, method;
    int m = 0, w = 0;
    double xi = 0, lb_time = 0, total_time = 0;
    uint64_t valid = 0, invalid = 0, pruned = 0, survivors = 0, matches = 0;
    bool has_lbip = false;
    double lbip_time = 0, lbip_rate = 0;
};

void emit_csv(const Row& r) {  // src/search_result.cpp:39-101
    const char* header =
        "dataset,normalization,metric,m,w,xi,method,lb_time,total_time,valid_candidates,"
        "invalid_candidates,pruned_candidates,pruning_rate,survivors,matches,"
        "lbip_time,lbip_pruning_rate,timestamp";
    const double rate = r.valid == 0 ? 0.0 : (double)r.pruned / (double)r.valid;
    std::string row = csv_escape(r.dataset) + (raw_mode() ? ",raw," : ",zscore,") + csv_escape(r.metric) + "," +
                      std::to_string(r.m) + "," + std::to_string(r.w) + "," + g17(r.xi) + "," +
                      csv_escape(r.method) + "," + g17(r.lb_time) + "," + g17(r.total_time) + "," +
                      std::to_string(r.valid) + "," + std::to_string(r.invalid) + "," +
                      std::to_string(r.pruned) + "," + g17(rate) + "," + std::to_string(r.survivors) +
                      "," + std::to_string(r.matches) + "," + (r.has_lbip ? g17(r.lbip_time) : "") + "," +
                      (r.has_lbip ? g17(r.lbip_rate) : "") + "," + timestamp_now();
    printf("EXPERIMENT_CSV_HEADER=%s\n", header);
    printf("EXPERIMENT_CSV=%s\n", row.c_str());
    fflush(stdout);
    const char* cfg = std::getenv("FSMELD_RESULTS_CSV");
    const std::string path = (cfg && *cfg) ? cfg : "experiment_results.csv";
    std::error_code ec;
    const bool need_header = !std::filesystem::exists(path, ec) || std::filesystem::file_size(path, ec) == 0;
    FILE* f = fopen(path.c_str(), "a");
    if (!f) {
        fprintf(stderr, "[Warning] Cannot append experiment CSV: %s\n", path.c_str());
        return;
    }
    if (need_header) fprintf(f, "%s\n", header);
    fprintf(f, "%s\n", row.c_str());
    fclose(f);
    printf("Experiment CSV saved to: %s\n", path.c_str());
}

struct Setup {
    fsmeld_ctx* ctx = nullptr;
    std::vector<double> q;
    long long n = 0;
    int m_k = 0;
    long long kml = 0, tsn = 0, forsize = 0, tail = 0;
};

int setup(const char* tp, const char* qp, int m, Setup* s) {
    int r = fsmeld_open_file(device_index(), tp, &s->ctx);
    if (r) {
        fprintf(stderr, "Error: %s\n", fsmeld_last_error(nullptr));
        return r;
    }
    s->n = fsmeld_target_length(s->ctx);
    if (raw_mode()) fsmeld_set_normalization(s->ctx, FSMELD_NORM_RAW);
    // FSMELD_TUNE_TABLE: a tuning table file (fsmeld_set_tuning) for the kernel
    // choices; by default the package's measured table beside the bin/ folder
    // of this executable, when present
    std::string table;
    if (const char* tp_env = std::getenv("FSMELD_TUNE_TABLE")) {
        table = tp_env;
    } else {
        char exe[4096];
        const ssize_t len = readlink("/proc/self/exe", exe, sizeof(exe) - 1);
        if (len > 0) {
            exe[len] = 0;
            std::string dir(exe);
            dir = dir.substr(0, dir.rfind('/'));         // .../bin
            table = dir.substr(0, dir.rfind('/')) + "/tune_table.txt";
        }
    }
    if (!table.empty()) {
        if (FILE* tf = fopen(table.c_str(), "r")) {
            std::string text;
            char buf[4096];
            size_t got;
            while ((got = fread(buf, 1, sizeof(buf), tf)) > 0) text.append(buf, got);
            fclose(tf);
            if (fsmeld_set_tuning(s->ctx, text.c_str()))
                fprintf(stderr, "[Warning] %s\n", fsmeld_last_error(s->ctx));
        }
    }
    if (!read_query(qp, m, &s->q)) {
        fprintf(stderr, "Error: Query must begin with m finite numeric values.\n");
        return FSMELD_E_ARG;
    }
    long long sel = 1;
    while (sel < 8LL * m) sel *= 2;
    if (s->n < sel) sel = s->n;
    s->m_k = (int)sel;
    s->kml = s->m_k - m + 1;
    s->tsn = s->n - m + 1;
    s->forsize = s->tsn / s->kml;
    s->tail = s->tsn % s->kml;
    return FSMELD_OK;
}

void print_geom(const Setup& s, int m) {
    printf("ts_n=%lld\nm=%d\nk_m_l=%lld\nm_k=%d\n", s.tsn, m, s.kml, s.m_k);
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" int fsmeld_search_file(const char* tp, const char* qp, int m, double cutoff, const char* tag, int w,
                                  double arg, int64_t eb, int64_t ee) {
    const double t0 = now_s();
    const int metric = metric_of(tag);
    if (!metric) { fprintf(stderr, "Error: Unsupported metric: %s\n", tag ? tag : ""); return FSMELD_E_ARG; }
    Setup s;
    int r = setup(tp, qp, m, &s);
    if (r) { fsmeld_close(s.ctx); return r; }
    if (s.n < 2LL * m - 1) { fsmeld_close(s.ctx); return FSMELD_OK; }  // src/fsmeld.cpp:615-617
    print_geom(s, m);
    printf("tail=%lld\nforsize=%lld\n", s.tail, s.forsize);
    std::vector<int64_t> idx(1 << 16), segc(3 * std::max<long long>(1, s.forsize));
    int64_t count = 0;
    fsmeld_counters cnt{};
    r = fsmeld_search(s.ctx, s.q.data(), m, cutoff, metric, w, arg, eb, ee, idx.data(), (int64_t)idx.size(), &count,
                      &cnt, segc.data());
    if (!r && count > (int64_t)idx.size()) {
        idx.resize(count);
        r = fsmeld_search(s.ctx, s.q.data(), m, cutoff, metric, w, arg, eb, ee, idx.data(), (int64_t)idx.size(),
                          &count, &cnt, segc.data());
    }
    if (r) {
        fprintf(stderr, "Error: %s\n", fsmeld_last_error(s.ctx));
        fsmeld_close(s.ctx);
        return r;
    }
    // progress lines (src/fsmeld.cpp:730-737): cumulative counters before segment ll
    const int fd100 = (int)(s.forsize / 100);
    unsigned long long k1 = 0, k2 = 0, k3 = 0;
    int pct = 0;
    for (long long ll = 0; ll < s.forsize; ++ll) {
        if (fd100 && ll % fd100 == 0) {
            printf("\b\b\b\b|%3d%%\n", pct++);
            printf("guolv=%g\n", (double)(k1 - k2) / k1);
            printf("guolv2=%g\n", (double)(k1 - k3) / k1);
        }
        k1 += segc[3 * ll];
        k2 += segc[3 * ll + 1];
        k3 += segc[3 * ll + 2];
    }
    const double total = now_s() - t0;
    const unsigned long long kk1 = cnt.valid, kk2 = cnt.after_lb, kk3 = cnt.after_glb;
    const double lb_rate = kk1 == 0 ? 0.0 : (double)(kk1 - kk2) / kk1;
    const double rate = kk1 == 0 ? 0.0 : (double)(kk1 - kk3) / kk1;
    const double lb_s = cnt.device_ms / 1000.0;
    printf("kk1=%llu\nkk2=%llu\nkk2=%llu\n", kk1, kk2, kk2);
    printf("Pruning Power (guolv)=%g\n", lb_rate);
    printf("Pruning Power (guolv2)=%g\n", rate);
    printf("LP_IP Lower Bound Time taken: %g ms\n", cnt.device_ms);
    printf("LP_IP Lower Bound Time taken: %g s\n", lb_s);
    printf("T_LB: %.17g s\n", lb_s);
    printf("T_total: %.17g s\n", total);
    printf("Invalid candidates: %lld\n", (long long)cnt.invalid);
    printf("Final dynamic threshold: %.17g\n", cutoff);
    printf("Total Valid Candidates: %llu\n", kk1);
    printf("Candidates after LP/IP: %llu\n", kk2);
    printf("Cascade: LB_IP+GLB+ELD\n");
    printf("Candidates after GLB: %llu\n", kk3);
    printf("Final Matches: %lld\n", (long long)count);
    if (!quiet_matches())
        for (int64_t i = 0; i < count; ++i) printf("A[%lld]=%lld\n", (long long)i, (long long)idx[i]);
    Row row;
    row.dataset = dataset_name(tp);
    row.metric = tag;
    row.method = "FSMELD";
    row.m = m; row.w = w; row.xi = cutoff;
    row.lb_time = lb_s; row.total_time = total;
    row.valid = kk1; row.invalid = cnt.invalid; row.pruned = kk1 - kk3; row.survivors = kk3;
    row.matches = count; row.has_lbip = true; row.lbip_time = lb_s; row.lbip_rate = lb_rate;
    emit_csv(row);
    fflush(stdout);
    fsmeld_close(s.ctx);
    return FSMELD_OK;
}

extern "C" int fsmeld_cutoff_file(const char* tp, const char* qp, int m, int k, const char* tag, int w, double arg,
                                  int64_t eb, int64_t ee) {
    const int metric = metric_of(tag);
    if (!metric) { fprintf(stderr, "Error: Unsupported metric: %s\n", tag ? tag : ""); return FSMELD_E_ARG; }
    Setup s;
    int r = setup(tp, qp, m, &s);
    if (r) { fsmeld_close(s.ctx); return r; }
    if (s.n < 2LL * m - 1) {
        fprintf(stderr, "Error: Target is too short for cutoff search.\n");
        fsmeld_close(s.ctx);
        return FSMELD_E_SHORT;
    }
    print_geom(s, m);
    std::vector<int64_t> idx(k);
    std::vector<double> dist(k);
    fsmeld_counters cnt{};
    r = fsmeld_cutoff(s.ctx, s.q.data(), m, k, metric, w, arg, eb, ee, idx.data(), dist.data(), &cnt);
    if (r) {
        fprintf(stderr, "Error: %s\n", fsmeld_last_error(s.ctx));
        fsmeld_close(s.ctx);
        return r;
    }
    const int fd100 = (int)(s.forsize / 100);
    int pct = 0;
    for (long long ll = 0; ll < s.forsize; ++ll) {
        if (fd100 && ll % fd100 == 0) {
            printf("\b\b\b\b|%3d%%\n", pct++);
            printf("Threshold=%.17g\n", cnt.threshold);
        }
    }
    const std::string bar(60, '=');
    printf("\n\n%s\n", bar.c_str());
    printf(" [FSMELD Top-K Threshold Results]\n");
    printf("  - Candidates checked by LB:   %lld\n", (long long)cnt.valid);
    printf("  - Pruned by LBIP:             %lld\n", (long long)(cnt.valid - cnt.after_lb));
    printf("  - Pruned by GLB:              %lld\n", (long long)(cnt.after_lb - cnt.after_glb));
    printf("  - Exact distances computed:   %lld\n", (long long)cnt.exact_evals);
    printf("  - Final Top-K Threshold:      %.17g\n", cnt.threshold);
    printf("%s\n\n", bar.c_str());
    for (int i = 0; i < k; ++i) printf("Rank %d: Index A[%d]=%lld\n", i + 1, i + 1, (long long)idx[i]);
    fflush(stdout);
    fsmeld_close(s.ctx);
    return FSMELD_OK;
}

extern "C" int fsmeld_exact_file(const char* tp, const char* qp, int m, double cutoff, const char* tag, int w,
                                 double arg, int64_t eb, int64_t ee) {
    const double t0 = now_s();
    const int metric = metric_of(tag);
    if (!metric) { fprintf(stderr, "Error: Unsupported metric: %s\n", tag ? tag : ""); return FSMELD_E_ARG; }
    Setup s;
    int r = setup(tp, qp, m, &s);
    if (r) { fsmeld_close(s.ctx); return r; }
    if (s.n < 2LL * m - 1) {
        fprintf(stderr, "Error: Target is too short for direct ELD scan.\n");
        fsmeld_close(s.ctx);
        return FSMELD_E_SHORT;
    }
    const bool quiet = quiet_matches();
    print_geom(s, m);
    printf("tail=%lld\nforsize=%lld\n", s.tail, s.forsize);
    std::vector<int64_t> idx(1 << 16);
    std::vector<double> dist(idx.size());
    int64_t count = 0;
    fsmeld_counters cnt{};
    r = fsmeld_exact(s.ctx, s.q.data(), m, cutoff, metric, w, arg, eb, ee, idx.data(), dist.data(),
                     (int64_t)idx.size(), &count, &cnt);
    if (!r && count > (int64_t)idx.size()) {
        idx.resize(count);
        dist.resize(count);
        r = fsmeld_exact(s.ctx, s.q.data(), m, cutoff, metric, w, arg, eb, ee, idx.data(), dist.data(),
                         (int64_t)idx.size(), &count, &cnt);
    }
    if (r) {
        fprintf(stderr, "Error: %s\n", fsmeld_last_error(s.ctx));
        fsmeld_close(s.ctx);
        return r;
    }
    // progress markers interleave with match lines in segment order (src/fsmeld.cpp:1173-1226)
    const int fd100 = (int)(s.forsize / 100);
    int pct = 0;
    long long next_ll = 0;
    auto progress_upto = [&](long long ll_end) {
        for (; next_ll < ll_end && next_ll < s.forsize; ++next_ll)
            if (fd100 && next_ll % fd100 == 0) printf("\b\b\b\b|%3d%% ", pct++);
    };
    for (int64_t i = 0; i < count; ++i) {
        const long long seg = std::min<long long>(idx[i] / s.kml, s.forsize);
        progress_upto(seg + 1);
        if (!quiet) printf("\nGET %s: %lf (index: %lld)\n", tag, dist[i], (long long)idx[i]);
    }
    progress_upto(s.forsize);
    printf("\n\n--- Statistics ---\n");
    printf("Total comparisons (kk1) = %lld\n", (long long)cnt.valid);
    printf("Exact ELD evaluations = %lld\n", (long long)cnt.exact_evals);
    printf("Final matches found: %lld\n", (long long)count);
    printf("Total Valid Candidates: %lld\n", (long long)cnt.valid);
    printf("Invalid candidates: %lld\n", (long long)cnt.invalid);
    printf("Exact ELD Evaluations: %lld\n", (long long)cnt.exact_evals);
    printf("Final Matches: %lld\n", (long long)count);
    if (!quiet)
        for (int64_t i = 0; i < count; ++i) printf("A[%lld] = %lld\n", (long long)i, (long long)idx[i]);
    const double total = now_s() - t0;
    printf("T_total: %.17g s\n", total);
    Row row;
    row.dataset = dataset_name(tp);
    row.metric = tag;
    row.method = "ELD";
    row.m = m; row.w = w; row.xi = cutoff;
    row.lb_time = 0.0; row.total_time = total;
    row.valid = cnt.valid; row.invalid = cnt.invalid; row.pruned = 0; row.survivors = cnt.valid;
    row.matches = count;
    emit_csv(row);
    fflush(stdout);
    fsmeld_close(s.ctx);
    return FSMELD_OK;
}
