// hrnn_dynamic_test: build on a split of the base set (or load a snapshot), build
// the mutable reverse lists, stream the rest in with insertPointDynamic, rebuild
// the flat reverse lists and measure recall -- the flags, split and report of the
// reference's src/hrnn_dynamic_test.cpp, with the index on the GPU
// (include/hrnn_b200.hpp).  The inserts of a batch reach the GPU together; the
// per-insert time is the batch time over its size.
#include <iomanip>
#include <memory>
#include <numeric>
#include <random>

#include "../../include/hrnn_b200.hpp"
#include "cli.hpp"

using HRNN = hnswlib::HRNN<float>;

namespace {

struct Eval {
    cli::Recall rc;
    double search_ms = 0;
};

Eval evaluate(HRNN& index, const cli::Fbin& query, const cli::RknnGt& gt, int m, int k, int ef) {
    index.setEf((size_t)ef);
    const uint32_t mm = (uint32_t)m, kp = (uint32_t)index.K_knng_, ee = (uint32_t)ef;
    auto t0 = cli::Clock::now();
    auto res = index.searchRknnBatch(query.data.data(), query.n, &mm, &kp, &ee, 1.0f, (size_t)k, true);
    Eval e;
    e.search_ms = cli::ms_since(t0);
    e.rc = cli::recall(gt, res, query.n);
    return e;
}

}  // namespace

int main(int argc, char* argv[]) try {
    std::string base_path, query_path, gt_path, snapshot_path, oracle_snapshot_path, precision;
    int batch_size_cli, M, ef_construction, K_knng, nn_iters, nn_sample, num_threads, k_rknn, m_proxy, ef_search;
    int m_update, bidirectional_flag, device;
    double split_ratio;
    cli::Options opt("HRNN Dynamic Update Test");
    opt.add("base", &base_path, "Base vectors (.fbin)", true)
        .add("query", &query_path, "Query vectors (.fbin)", true)
        .add("gt", &gt_path, "RkNN groundtruth of the full base set", true)
        .add("snapshot", &snapshot_path, "Index snapshot of the initial split (loaded if present, else saved)",
             false, std::string(""))
        .add("oracle_snapshot", &oracle_snapshot_path, "Index built on all points, for the recall gap", false,
             std::string(""))
        .add("batch_size", &batch_size_cli, "Points to insert (0 = all the rest)", false, 0)
        .add("M", &M, "HNSW M parameter", false, 16)
        .add("ef_construction", &ef_construction, "HNSW ef_construction", false, 200)
        .add("K_knng", &K_knng, "KNNG depth", false, 500)
        .add("nn_iters", &nn_iters, "NNDescent iterations", false, 3)
        .add("nn_sample", &nn_sample, "NNDescent sample size", false, 20)
        .add("num_threads", &num_threads, "Host threads (accepted; the work runs on the GPU)", false, 64)
        .add("k", &k_rknn, "RkNN k", false, 10)
        .add("m", &m_proxy, "Proxies of the evaluation search", false, 50)
        .add("ef_search", &ef_search, "HNSW ef_search", false, 200)
        .add("split", &split_ratio, "Fraction of the base set built up front", false, 0.5)
        .add("m_update", &m_update, "Proxies of the insert's self-query (0 = all neighbours)", false, 0)
        .add("bidirectional", &bidirectional_flag, "Refresh the new point's own list too (0/1)", false, 0)
        .add("precision", &precision, "Search precision: fp32 or bf16", false, std::string("fp32"))
        .add("device", &device, "CUDA device", false, 0);
    if (!opt.parse(argc, argv)) return 0;

    std::cout << "=== HRNN Dynamic Update Test (B200) ===" << std::endl;
    std::cout << "  M=" << M << "  ef_construction=" << ef_construction << "  K_knng=" << K_knng << std::endl;
    std::cout << "  split=" << split_ratio << "  k=" << k_rknn << "  m=" << m_proxy << "  ef_search=" << ef_search
              << "  m_update=" << m_update << "  bidirectional=" << bidirectional_flag << std::endl;

    auto t0 = cli::Clock::now();
    std::cout << "\n[1] Loading base / query / GT" << std::endl;
    auto base = cli::load_fbin(base_path);
    auto query = cli::load_fbin(query_path);
    auto gt = cli::load_rknn_gt(gt_path);
    std::cout << "      n=" << base.n << "  d=" << base.d << "  nq=" << query.n << "  (" << (long)cli::ms_since(t0)
              << " ms)" << std::endl;

    // The split of src/hrnn_dynamic_test.cpp:200-203: a std::mt19937(42) shuffle.
    const size_t n = base.n;
    const size_t split_n = (size_t)((double)n * split_ratio);
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    std::mt19937 rng(42);
    std::shuffle(perm.begin(), perm.end(), rng);
    const size_t insert_total = n - split_n;
    const size_t batch_n = batch_size_cli > 0 ? std::min<size_t>((size_t)batch_size_cli, insert_total) : insert_total;
    std::cout << "\n[2] Split: initial=" << split_n << "  incremental_total=" << insert_total
              << "  active_batch=" << batch_n << std::endl;

    hnswlib::L2Space space(base.d);
    std::unique_ptr<HRNN> index;
    double build_ms = 0;
    std::ifstream probe(snapshot_path);
    if (!snapshot_path.empty() && probe.good()) {
        std::cout << "\n[3] Loading snapshot: " << snapshot_path << std::endl;
        t0 = cli::Clock::now();
        index = std::make_unique<HRNN>(&space, snapshot_path, false, n, device);
        const double load_ms = cli::ms_since(t0);
        std::cout << "      Loaded (" << (long)load_ms << " ms)  cur_elements=" << index->getCurrentElementCount()
                  << "  K_knng=" << index->K_knng_ << "  knng_built=" << index->knng_built_ << std::endl;
        t0 = cli::Clock::now();
        index->buildRKNNG_mutable();
        build_ms = load_ms + cli::ms_since(t0);
    } else {
        std::cout << "\n[3] Building HRNN on initial " << split_n << " points" << std::endl;
        index = std::make_unique<HRNN>(&space, n, M, ef_construction, 100, false, (size_t)K_knng, device);
        t0 = cli::Clock::now();
        for (size_t i = 0; i < split_n; ++i)
            index->addPoint(base.data.data() + (size_t)perm[i] * base.d, (hnswlib::labeltype)perm[i]);
        index->getCurrentElementCount();
        const double hnsw_ms = cli::ms_since(t0);
        std::cout << "      HNSW + initial KNNG: " << (long)hnsw_ms << " ms" << std::endl;
        t0 = cli::Clock::now();
        index->refineKNNG(nn_iters, nn_sample);
        const double refine_ms = cli::ms_since(t0);
        std::cout << "      Refine: " << (long)refine_ms << " ms" << std::endl;
        if (!snapshot_path.empty()) {
            std::cout << "\n[3s] Saving snapshot to " << snapshot_path << std::endl;
            index->saveIndex(snapshot_path);
        }
        t0 = cli::Clock::now();
        index->buildRKNNG_mutable();
        const double rk_ms = cli::ms_since(t0);
        std::cout << "      RKNNG: " << (long)rk_ms << " ms" << std::endl;
        build_ms = hnsw_ms + refine_ms + rk_ms;
    }
    std::cout << "\n      Total initial build/load: " << (long)build_ms << " ms" << std::endl;

    std::cout << "\n[4] Inserting " << batch_n << " points incrementally" << std::endl;
    t0 = cli::Clock::now();
    for (size_t i = 0; i < batch_n; ++i) {
        const uint32_t id = perm[split_n + i];
        index->insertPointDynamic(base.data.data() + (size_t)id * base.d, (hnswlib::labeltype)id,
                                  (unsigned)m_update, bidirectional_flag != 0);
    }
    const size_t after = index->getCurrentElementCount();  // the queued inserts run here
    const double maint_ms = cli::ms_since(t0);
    const double per_insert = batch_n ? maint_ms / (double)batch_n : 0.0;
    std::cout << "      Total insert: " << (long)maint_ms << " ms" << std::endl;
    std::cout << "      Per-insert: " << std::fixed << std::setprecision(3) << per_insert << " ms" << std::endl;
    std::cout << "      Index size after maintenance: " << after << std::endl;

    std::cout << "\n[5] Searching (m=" << m_proxy << ", threshold=1, ef_search=" << ef_search << ")" << std::endl;
    t0 = cli::Clock::now();
    index->buildRKNNG();
    std::cout << "      Flat RKNNG for search: " << (long)cli::ms_since(t0) << " ms" << std::endl;
    index->setPrecision(precision == "bf16" ? HRNN_PREC_BF16 : HRNN_PREC_FP32_EXACT);
    Eval ev = evaluate(*index, query, gt, m_proxy, k_rknn, ef_search);
    std::cout << std::fixed << std::setprecision(6);
    std::cout << "      Macro Recall = " << ev.rc.macro << std::endl;
    std::cout << "      Micro Recall = " << ev.rc.micro << std::endl;
    std::cout << std::fixed << std::setprecision(2);
    std::cout << "      Avg results/query = " << ev.rc.avg_results << std::endl;
    std::cout << "      Search time = " << (long)ev.search_ms << " ms ("
              << (double)query.n * 1000.0 / std::max(1e-3, ev.search_ms) << " QPS)" << std::endl;

    bool has_oracle = false;
    Eval oe;
    if (!oracle_snapshot_path.empty()) {
        std::cout << "\n[6] Loading oracle snapshot: " << oracle_snapshot_path << std::endl;
        HRNN oracle(&space, oracle_snapshot_path, false, n, device);
        oracle.buildRKNNG();
        oracle.setPrecision(precision == "bf16" ? HRNN_PREC_BF16 : HRNN_PREC_FP32_EXACT);
        oe = evaluate(oracle, query, gt, m_proxy, k_rknn, ef_search);
        has_oracle = true;
        std::cout << std::fixed << std::setprecision(6);
        std::cout << "      Oracle Macro Recall = " << oe.rc.macro << std::endl;
        std::cout << "      Oracle Micro Recall = " << oe.rc.micro << std::endl;
    }

    std::cout << "\n=== Summary ===" << std::endl;
    std::cout << "  Initial build/load (" << split_n << " pts): " << (long)build_ms << " ms" << std::endl;
    std::cout << "  Maintained batch size: " << batch_n << std::endl;
    std::cout << "  Maintenance time: " << (long)maint_ms << " ms" << std::endl;
    std::cout << "  Per-insert latency: " << std::fixed << std::setprecision(3) << per_insert << " ms" << std::endl;
    std::cout << "  Macro Recall = " << std::fixed << std::setprecision(6) << ev.rc.macro << std::endl;
    std::cout << "  Micro Recall = " << std::fixed << std::setprecision(6) << ev.rc.micro << std::endl;
    if (has_oracle) {
        std::cout << "  Oracle macro gap = " << std::fixed << std::setprecision(6) << (ev.rc.macro - oe.rc.macro)
                  << std::endl;
        std::cout << "  Oracle micro gap = " << std::fixed << std::setprecision(6) << (ev.rc.micro - oe.rc.micro)
                  << std::endl;
    }
    return 0;
} catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
}
