// hrnn_search: RkNN search sweep over m and score thresholds with recall against
// a ground-truth file -- the flags and report of the reference's
// src/hrnn_search.cpp, with the search on the GPU (include/hrnn_b200.hpp).
//
// Additional flags: --batch (queries per device call; 1 times each query alone
// as the reference does, 0 sends all queries in one call), --precision (fp32:
// the reference's answers; bf16: the mixed-precision form, exact decisions) and
// --device.
#include <iomanip>
#include <memory>

#include "../../include/hrnn_b200.hpp"
#include "cli.hpp"

namespace {

struct Lat {
    double mean = 0, p50 = 0, p95 = 0, p99 = 0, max = 0;
};

Lat latency(std::vector<double> t) {
    Lat s;
    if (t.empty()) return s;
    std::sort(t.begin(), t.end());
    double tot = 0;
    for (double x : t) tot += x;
    s.mean = tot / (double)t.size();
    auto pct = [&](double p) {  // linear interpolation between ranks
        const double r = p * (double)(t.size() - 1);
        const size_t lo = (size_t)std::floor(r), hi = (size_t)std::ceil(r);
        return t[lo] + (t[hi] - t[lo]) * (r - (double)lo);
    };
    s.p50 = pct(0.50);
    s.p95 = pct(0.95);
    s.p99 = pct(0.99);
    s.max = t.back();
    return s;
}

}  // namespace

int main(int argc, char* argv[]) try {
    std::string index_path, query_path, gt_path, m_str, threshold_str, precision;
    int k, K_prime, ef_search, max_queries, max_k_serve, batch, device;
    cli::Options opt("HRNN Search Options");
    opt.add("index_path", &index_path, "HRNN index path", true)
        .add("query", &query_path, "Query vectors (.fbin)", true)
        .add("gt", &gt_path, "RkNN groundtruth file", true)
        .add("k", &k, "RkNN k parameter", false, 10)
        .add("K_prime", &K_prime, "KNNG K' truncation (use first K' reverse entries)", false, 500)
        .add("m", &m_str, "Proxy counts to sweep (comma-separated)", false, std::string("1,3,5,10,20,50"))
        .add("threshold,t", &threshold_str, "Binary score thresholds (comma-separated)", false, std::string("1"))
        .add("ef_search", &ef_search, "HNSW ef_search", false, 200)
        .add("max_queries", &max_queries, "0=all", false, 0)
        .add("max_k_serve", &max_k_serve, "Enable serve mode for k<=max_k_serve (0=off)", false, 0)
        .add("batch", &batch, "Queries per device call (0 = all, 1 = one at a time)", false, 0)
        .add("precision", &precision, "fp32 (reference answers) or bf16 (mixed precision)", false,
             std::string("fp32"))
        .add("device", &device, "CUDA device", false, 0);
    if (!opt.parse(argc, argv)) return 0;

    std::vector<int> m_values;
    for (auto& s : cli::split(m_str)) m_values.push_back(std::stoi(s));
    if (m_values.empty()) m_values.push_back(20);
    std::vector<float> thresholds;
    for (auto& s : cli::split(threshold_str)) thresholds.push_back(std::stof(s));
    if (thresholds.empty()) thresholds.push_back(1.0f);
    if (precision != "fp32" && precision != "bf16") throw std::runtime_error("--precision must be fp32 or bf16");

    std::cout << "=== HRNN RkNN Search (B200) ===" << std::endl;
    std::cout << "  k=" << k << "  K'=" << K_prime << "  ef_search=" << ef_search << "  precision=" << precision
              << std::endl;
    std::cout << "  m values:";
    for (int m : m_values) std::cout << " " << m;
    std::cout << std::endl << "  thresholds:";
    for (float t : thresholds) std::cout << " " << t;
    std::cout << std::endl;

    std::cout << "\n[1] Loading queries " << query_path << std::endl;
    auto query = cli::load_fbin(query_path);
    std::cout << "      nq=" << query.n << "  d=" << query.d << std::endl;
    std::cout << "[2] Loading RkNN GT " << gt_path << std::endl;
    auto gt = cli::load_rknn_gt(gt_path);
    std::cout << "      nq=" << gt.nq << "  total=" << gt.off.back() << std::endl;
    std::cout << "[3] Loading HRNN index " << index_path << std::endl;
    auto t0 = cli::Clock::now();
    hnswlib::L2Space space(query.d);
    auto index = std::make_unique<hnswlib::HRNN<float>>(&space, index_path, false, 0, device);
    index->setEf((size_t)ef_search);
    index->setPrecision(precision == "bf16" ? HRNN_PREC_BF16 : HRNN_PREC_FP32_EXACT);
    std::cout << "      Done (" << (long)cli::ms_since(t0) << " ms)" << std::endl;
    std::cout << "      K_knng=" << index->K_knng_ << "  knng_built=" << index->knng_built_
              << "  rknng_built=" << index->rknng_built_ << std::endl;
    if (max_k_serve > 0) {
        std::cout << "[3b] Compacting for serve mode (max_k_serve=" << max_k_serve << ")" << std::endl;
        auto tc = cli::Clock::now();
        index->compactForServing((size_t)max_k_serve);
        std::cout << "      Done (" << (long)cli::ms_since(tc) << " ms)" << std::endl;
    }

    size_t nq = query.n;
    if (max_queries > 0) nq = std::min<size_t>((size_t)max_queries, query.n);
    const size_t bs = batch <= 0 ? std::max<size_t>(nq, 1) : (size_t)batch;
    for (int m : m_values) {
        for (float threshold : thresholds) {
            std::cout << "\n[4] Search: nq=" << nq << "  m=" << m << "  threshold=" << threshold << std::endl;
            std::vector<std::vector<hnswlib::labeltype>> results;
            results.reserve(nq);
            std::vector<double> call_ms;
            const uint32_t mm = (uint32_t)m, kp = (uint32_t)K_prime, ee = (uint32_t)ef_search;
            for (size_t q0 = 0; q0 < nq; q0 += bs) {
                const size_t c = std::min(bs, nq - q0);
                auto ta = cli::Clock::now();
                auto r = index->searchRknnBatch(query.data.data() + q0 * query.d, c, &mm, &kp, &ee, threshold,
                                                (size_t)k, true);
                call_ms.push_back(cli::ms_since(ta));
                for (auto& x : r) results.push_back(std::move(x));
            }
            if (nq == query.n) {
                auto rc = cli::recall(gt, results, nq);
                std::cout << "      Macro Recall = " << std::fixed << std::setprecision(6) << rc.macro << std::endl;
                std::cout << "      Micro Recall = " << std::fixed << std::setprecision(6) << rc.micro << std::endl;
            }
            double avg = 0;
            for (auto& r : results) avg += (double)r.size();
            std::cout << "      Avg results/query = " << std::fixed << std::setprecision(2) << avg / (double)nq
                      << std::endl;
            auto ls = latency(call_ms);
            std::cout << std::fixed << std::setprecision(3);
            std::cout << "      Latency per call of " << bs << " (ms): mean=" << ls.mean << "  p50=" << ls.p50
                      << "  p95=" << ls.p95 << "  p99=" << ls.p99 << "  max=" << ls.max << std::endl;
            double total = 0;
            for (double t : call_ms) total += t;
            std::cout << "      QPS = " << std::fixed << std::setprecision(2) << (double)nq * 1000.0 / total
                      << std::endl;
        }
    }
    return 0;
} catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
}
