// psm_match: drop-in for the reference's SubgraphMatching.out command line.
//
// Accepts the reference's flags (matching/matchingcommand.cpp:5-27, defaults
// matching/matchingcommand.h:70-159) and appends the same log block per
// (thread count, method) pair to -OutputFile, each line prefixed
// "[Thread 1] " like utility/statistics/Logs.h:88-96. The C-mode driver loop
// mirrors split_C_test (matching/StudyPerformance.cpp:1039-1781): for every
// entry of -threadnums and every FILTER_ORDER_ENGINE triple of -BackMethods,
// one query run and one log block. Q mode (-QorCandi Q, split_Q_test,
// StudyPerformance.cpp:100-1037) runs the decomposition + hash-join path
// (psm_match_join_ex) with the -Qpattern decomposition (STAR, the default,
// TWINTWIG, SEED, SKETCHTREE; also this library's BOUNDED and COST, whose
// units have at most -max_unit vertices, default 12) and the -JoinMethod
// paradigm (LEFTDEEP, the default, or BUSHY); -max_unit also splits STAR's
// stars. The count does not depend on the decomposition.
//
// Differences a caller can see:
//  - every engine name is accepted and served by the set-intersection
//    enumerator (all of the reference's engines count the same embeddings);
//    filters other than NLF / GQL / CFL and orders other than GQL / CFL are
//    rejected with the reference's "is not supported" line and exit 1;
//  - -threadnums values are recorded in the log but do not change the device
//    execution;
//  - filtering, table building and ordering run fused in one device launch:
//    "Preprocessing time" is their measured sum and the three per-stage lines
//    print 0; "Host Wall Time" is an added line (the call's wall time);
//  - paths with fewer slashes than the reference's extract_graph_file
//    (StudyPerformance.cpp:66-83) needs are printed whole instead of aborting;
//  - without -OutputFile the log goes to stdout.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "psm_b200.h"

namespace {

struct Flags {
    std::map<std::string, std::string> kv;
    std::string get(const std::string& k, const std::string& def) const {
        auto it = kv.find(k);
        return it == kv.end() || it->second.empty() ? def : it->second;
    }
    bool has(const std::string& k) const {
        auto it = kv.find(k);
        return it != kv.end() && !it->second.empty();
    }
};

// Same lookup as the reference's CommandParser: the token after the key.
Flags parse_flags(int argc, char** argv) {
    static const char* keys[] = {"-a", "-i", "-q", "-d", "-d0", "-w0", "-filter", "-order", "-engine", "-num",
                                 "-time_limit", "-order_num", "-dis_file", "-csr", "-OutputFile", "-threadnums",
                                 "-split", "-schedule", "-QorCandi", "-Qpattern", "-JoinMethod", "-BackMethods",
                                 "-device", "-arena_gb", "-max_unit"};
    Flags f;
    for (int i = 1; i + 1 < argc; ++i)
        for (const char* k : keys)
            if (std::string(argv[i]) == k) f.kv[k] = argv[i + 1];
    return f;
}

std::vector<std::string> split(const std::string& s, char sep) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, sep)) out.push_back(tok);
    return out;
}

// Last `num` path components (the reference's extract_graph_file), or the
// whole path when it has fewer slashes.
std::string tail_components(const std::string& path, int num) {
    size_t pos = path.size();
    for (int i = 0; i < num; ++i) {
        if (pos == 0) return path;
        size_t p = path.rfind('/', pos - 1);
        if (p == std::string::npos) return path;
        pos = p;
    }
    return path.substr(pos + 1);
}

// Query graph in the reference text format ("t V E", "v id label deg",
// "e u v"; graph/graph.cpp:92-172).
bool load_query(const std::string& path, std::vector<uint32_t>& labels, std::vector<uint32_t>& edges,
                std::string& err) {
    std::ifstream in(path);
    if (!in) {
        err = "cannot open query file " + path;
        return false;
    }
    std::string tag;
    uint32_t V = 0;
    uint64_t E = 0;
    while (in >> tag) {
        if (tag == "t") {
            in >> V >> E;
            labels.assign(V, 0);
        } else if (tag == "v") {
            uint32_t id, lab, deg;
            in >> id >> lab >> deg;
            if (id >= V) {
                err = "vertex id out of range in " + path;
                return false;
            }
            labels[id] = lab;
        } else if (tag == "e") {
            uint32_t a, b;
            in >> a >> b;
            std::string rest;
            std::getline(in, rest);  // an optional edge label is ignored, as by the reference
            if (a >= V || b >= V) {
                err = "edge endpoint out of range in " + path;
                return false;
            }
            edges.push_back(a);
            edges.push_back(b);
        } else {
            std::string rest;
            std::getline(in, rest);
        }
    }
    if (V == 0) {
        err = "empty query graph " + path;
        return false;
    }
    return true;
}

struct Log {
    std::ostream* os;
    template <class T>
    Log& operator<<(const T& x) {
        line << x;
        return *this;
    }
    void end() {
        *os << "[Thread 1] " << line.str() << "\n";
        line.str("");
        line.clear();
    }
    std::ostringstream line;
};

double ns_to_s(double ns) { return ns / 1e9; }

}  // namespace

int main(int argc, char** argv) {
    Flags f = parse_flags(argc, argv);
    const std::string qpath = f.get("-q", ""), dpath = f.get("-d", "");
    const std::string mode = f.get("-QorCandi", "NOSPLIT");
    const std::string out_path = f.get("-OutputFile", "");
    std::ofstream file;
    std::ostream* os = &std::cout;
    if (!out_path.empty()) {
        file.open(out_path, std::ios::out | std::ios::app);
        if (!file) {
            std::cout << "Error: Failed to open log file at " << out_path << std::endl;
            return 1;
        }
        os = &file;
    }
    Log log{os};
    if (mode != "C" && mode != "Q") {
        log << "Error: The split mode is not defined.";
        log.end();
        return 1;
    }
    if (qpath.empty() || dpath.empty()) {
        std::cerr << "usage: psm_match -d <data graph> -q <query graph> -QorCandi C|Q [reference flags] "
                     "[-device i] [-arena_gb g] [-max_unit k]\n";
        return 2;
    }
    const std::string num = f.get("-num", "MAX"), tl = f.get("-time_limit", "60");
    const std::string split_type = f.get("-split", "shixuan"), schedule = f.get("-schedule", "steal");
    const std::vector<std::string> threads = split(f.get("-threadnums", "1"), ',');
    const std::vector<std::string> methods = split(f.get("-BackMethods", "DPiso"), ',');
    const int device = std::atoi(f.get("-device", "0").c_str());
    const double arena_gb = std::atof(f.get("-arena_gb", "16").c_str());
    const bool have_max_unit = f.has("-max_unit");
    const uint32_t max_unit = (uint32_t)std::atoi(f.get("-max_unit", "12").c_str());
    const std::string qpattern = f.get("-Qpattern", "STAR"), join_method = f.get("-JoinMethod", "LEFTDEEP");
    psm_join_options jo{PSM_SPLIT_STAR, PSM_JOIN_LEFTDEEP, have_max_unit ? max_unit : 0u, 0};
    if (mode == "Q") {
        if (qpattern == "STAR") jo.pattern = PSM_SPLIT_STAR;
        else if (qpattern == "TWINTWIG") jo.pattern = PSM_SPLIT_TWINTWIG;
        else if (qpattern == "SEED") jo.pattern = PSM_SPLIT_SEED;
        else if (qpattern == "SKETCHTREE") jo.pattern = PSM_SPLIT_SKETCHTREE;
        else if (qpattern == "BOUNDED") jo.pattern = PSM_SPLIT_BOUNDED, jo.max_unit = max_unit;
        else if (qpattern == "COST") jo.pattern = PSM_SPLIT_COST, jo.max_unit = max_unit;
        else {
            log << "Error: The split pattern '" << qpattern << "' is not defined."; log.end();
            return 1;
        }
        if (join_method == "LEFTDEEP") jo.join_method = PSM_JOIN_LEFTDEEP;
        else if (join_method == "BUSHY") jo.join_method = PSM_JOIN_BUSHY;
        else {
            log << "Error: The join method '" << join_method << "' is not defined."; log.end();
            return 1;
        }
    }

    auto t0 = std::chrono::steady_clock::now();
    psm_graph* g = nullptr;
    if (psm_graph_load(dpath.c_str(), &g) != PSM_OK) {
        std::cerr << "psm_match: " << psm_last_error() << "\n";
        return 1;
    }
    std::vector<uint32_t> qlab, qedges;
    std::string err;
    if (!load_query(qpath, qlab, qedges, err)) {
        std::cerr << "psm_match: " << err << "\n";
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    const double load_ns = (double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count();
    psm_context* ctx = nullptr;
    if (psm_context_create(device, (uint64_t)(arena_gb * (1ull << 30)), &ctx) != PSM_OK) {
        std::cerr << "psm_match: " << psm_last_error() << "\n";
        return 1;
    }
    psm_query_desc q{(uint32_t)qlab.size(), (uint32_t)(qedges.size() / 2), qlab.data(), qedges.data()};
    int64_t output_limit = std::numeric_limits<int64_t>::max();
    if (num != "MAX") output_limit = std::atoll(num.c_str());
    const double time_limit = std::atof(tl.c_str());

    int exit_code = 0;
    for (const std::string& nt : threads) {
        for (const std::string& m : methods) {
            std::vector<std::string> p = split(m, '_');
            p.resize(3);
            const std::string& ft = p[0];
            const std::string& ot = p[1];
            const std::string& et = p[2];
            log << "Start the query"; log.end();
            log << "Input Query Graph File: " << qpath; log.end();
            log << "Input Data Graph File: " << tail_components(dpath, 3); log.end();
            log << "Maximum Embedding Number: " << num; log.end();
            log << "Time Limit: " << tl; log.end();
            log << "Num Threads: " << nt; log.end();
            if (mode == "C") {
                log << "Split Type: " << split_type; log.end();
                log << "Schedule Type: " << schedule; log.end();
            } else {
                log << "QuerySplit Pattern: " << qpattern; log.end();
                log << "Join Paradigm: " << join_method; log.end();
            }
            log << "Filter Type: " << ft; log.end();
            log << "Order Type: " << ot; log.end();
            log << "Engine Type: " << et; log.end();
            log << "Output Limit: " << output_limit; log.end();
            psm_options opt{};
            if (ft == "NLF") opt.filter = PSM_FILTER_NLF;
            else if (ft == "GQL") opt.filter = PSM_FILTER_GQL;
            else if (ft == "CFL") opt.filter = PSM_FILTER_CFL;
            else {
                log << "The specified filter type '" << ft << "' is not supported."; log.end();
                exit_code = 1;
                continue;
            }
            if (ot == "GQL") opt.order = PSM_ORDER_GQL;
            else if (ot == "CFL") opt.order = PSM_ORDER_CFL;
            else {
                log << "The specified order type '" << ot << "' is not supported."; log.end();
                exit_code = 1;
                continue;
            }
            opt.engine = et == "GQL" ? PSM_ENGINE_GQL : et == "EXPLORE" ? PSM_ENGINE_EXPLORE : PSM_ENGINE_LFTJ;
            opt.cap = num == "MAX" ? 0 : (uint64_t)output_limit;
            opt.time_limit_s = time_limit;
            log << "-----"; log.end();
            log << "Build indices..."; log.end();
            log << "-----"; log.end();
            log << "Generate a matching order..."; log.end();
            psm_result r{};
            psm_join_result jr{};
            auto w0 = std::chrono::steady_clock::now();
            int rc = mode == "C" ? psm_match(ctx, g, &q, &opt, &r) : psm_match_join_ex(ctx, g, &q, &opt, &jo, &jr);
            auto w1 = std::chrono::steady_clock::now();
            if (rc != PSM_OK && rc != PSM_ERR_TIMEOUT) {
                std::cerr << "psm_match: " << psm_status_string(rc) << ": " << psm_last_error() << "\n";
                exit_code = 1;
                continue;
            }
            double join_s = 0;
            if (mode == "Q") {
                // the join path's figures in the plain path's fields
                r.count = jr.count;
                r.prep_ms = jr.prep_ms;
                r.enum_ms = jr.enum_ms;
                r.memory_bytes = jr.memory_bytes;
                r.overtime = rc == PSM_ERR_TIMEOUT;
                join_s = jr.join_ms / 1e3;
                log << "subgraph count == " << jr.units; log.end();
                for (uint32_t k = 0; k < jr.units; ++k) {
                    log << "subgraph " << k << " vertices count == " << __builtin_popcount(jr.unit_mask[k]); log.end();
                }
            } else {
                log << "subgraph count == 1"; log.end();
                log << "subgraph 0 vertices count == " << q.num_vertices; log.end();
            }
            log << "-----"; log.end();
            log << "Enumerate..."; log.end();
            log << "schedule_type == " << schedule; log.end();
            log << "split_type == " << split_type; log.end();
            const double prep_s = r.prep_ms / 1e3, enum_s = r.enum_ms / 1e3;
            const double wall_s = ns_to_s((double)std::chrono::duration_cast<std::chrono::nanoseconds>(w1 - w0).count());
            log << "InitTasks time: " << 0; log.end();
            log << "Load graphs time (seconds): " << ns_to_s(load_ns); log.end();
            log << "Build table time (seconds): " << 0; log.end();
            log << "Filter vertices time (seconds): " << 0; log.end();
            log << "Split Qeury Pattern Time: " << 0; log.end();
            log << "Generate query plan time (seconds): " << 0; log.end();
            log << "Enumerate time (seconds): " << enum_s; log.end();
            log << "Preprocessing time (seconds): " << prep_s; log.end();
            log << "Join time (seconds): " << join_s; log.end();
            log << "Total time (seconds): " << prep_s + enum_s + join_s; log.end();
            log << "Memory cost (MB): " << r.memory_bytes / (double)(1024 * 1024); log.end();
            log << "#Embeddings: " << r.count; log.end();
            log << "Call Count: " << r.calls; log.end();
            log << "Thread Enum Time: " << enum_s; log.end();
            log << "Thread Execution Time: " << enum_s; log.end();
            log << "Thread Split Time: " << 0; log.end();
            log << "Thread Idle Time: " << 0; log.end();
            log << "Thread Call Count: " << r.calls; log.end();
            log << "Thread Embedding Count: " << r.count; log.end();
            log << "TaskNum: " << r.tasks; log.end();
            log << "Per Call Time (nanoseconds): " << (uint64_t)(r.enum_ms * 1e6 / (r.calls ? r.calls : 1)); log.end();
            log << "Overtime: " << r.overtime; log.end();
            log << "Host Wall Time (seconds): " << wall_s; log.end();
            log << "End the query"; log.end();
        }
    }
    psm_context_free(ctx);
    psm_graph_free(g);
    return exit_code;
}
