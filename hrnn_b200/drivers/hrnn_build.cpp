// hrnn_build: HNSW insertion with the KNN-graph seed, NNDescent refinement,
// reverse-KNN CSR, .idx save -- the steps and flags of the reference's
// src/hrnn_build.cpp, with the index on the GPU (include/hrnn_b200.hpp).
#include <atomic>
#include <iomanip>
#include <memory>

#include "../../include/hrnn_b200.hpp"
#include "cli.hpp"

int main(int argc, char* argv[]) try {
    std::string base_path, index_path;
    int M, ef_construction, K_knng, nn_iters, nn_sample, num_threads, device;
    cli::Options opt("HRNN Build Options");
    opt.add("base", &base_path, "Path to base vectors (.fbin)", true)
        .add("index_path", &index_path, "Index path to save", true)
        .add("M", &M, "HNSW M parameter", false, 16)
        .add("ef_construction", &ef_construction, "HNSW ef_construction parameter", false, 200)
        .add("K_knng", &K_knng, "KNNG depth (K nearest neighbors to store per node)", false, 500)
        .add("nn_iters", &nn_iters, "NNDescent refinement iterations", false, 3)
        .add("nn_sample", &nn_sample, "NNDescent sample size per node per iteration", false, 20)
        .add("num_threads", &num_threads, "Number of host threads (accepted; the work runs on the GPU)", false, 64)
        .add("device", &device, "CUDA device", false, 0);
    if (!opt.parse(argc, argv)) return 0;

    std::cout << "=== HRNN Index Build (B200) ===" << std::endl;
    std::cout << "  M=" << M << "  ef_construction=" << ef_construction << "  K_knng=" << K_knng << std::endl;
    std::cout << "  nn_iters=" << nn_iters << "  nn_sample=" << nn_sample << std::endl;

    std::cout << "\n[1] Loading base  " << base_path << std::endl;
    auto t0 = cli::Clock::now();
    auto base = cli::load_fbin(base_path);
    std::cout << "      n=" << base.n << "  d=" << base.d << "  (" << (long)cli::ms_since(t0) << " ms)" << std::endl;

    std::cout << "\n[2] Building HNSW + initial KNNG ..." << std::endl;
    hnswlib::L2Space space(base.d);
    auto index = std::make_unique<hnswlib::HRNN<float>>(&space, base.n, M, ef_construction, 100, false,
                                                         (size_t)K_knng, device);
    t0 = cli::Clock::now();
    for (uint32_t i = 0; i < base.n; ++i)
        index->addPoint(base.data.data() + (size_t)i * base.d, (hnswlib::labeltype)i);
    const size_t n_done = index->getCurrentElementCount();  // the queued points go to the GPU here
    std::cout << "      HNSW addPoint: " << n_done << " / " << base.n << std::endl;
    std::cout << "      HNSW + initial KNNG done  (" << (long)cli::ms_since(t0) << " ms)" << std::endl;

    std::cout << "\n[3] Refining KNNG (NNDescent local join, " << nn_iters << " iterations) ..." << std::endl;
    t0 = cli::Clock::now();
    index->refineKNNG(nn_iters, nn_sample);
    std::cout << "      Refine done  (" << (long)cli::ms_since(t0) << " ms)" << std::endl;

    std::cout << "\n[4] Building RKNNG (CSR transpose) ..." << std::endl;
    t0 = cli::Clock::now();
    index->buildRKNNG();
    std::cout << "      RKNNG done  (" << (long)cli::ms_since(t0) << " ms)" << std::endl;

    std::cout << "\n[5] Saving index to " << index_path << std::endl;
    t0 = cli::Clock::now();
    index->saveIndex(index_path);
    std::cout << "      Saved  (" << (long)cli::ms_since(t0) << " ms)" << std::endl;
    return 0;
} catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
}
