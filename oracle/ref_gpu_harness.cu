// ref_gpu_harness.cu -- C entry points over the reference's OWN CUDA path.
//
// TEST INFRASTRUCTURE ONLY.  Built by `make -C oracle refgpu REF=<dir>`
// against the reference sources where they lie; the library goes to
// oracle/_ref/ and is never committed.  It is the plain one-configuration-
// per-launch GPU form of the reference, timed beside the engine.
//
// The reference's driver (cuckoo_bench.cu, with gpu_shared.cuh, gpu_cached.cuh,
// cuckoo_core.hpp and checkpoint.hpp) is compiled unmodified; only its `main`
// is renamed so that this file can provide the library's entry points.
// ref_gpu_run() calls the reference's stock worker, gpu_worker()
// (cuckoo_bench.cu:813-1038): its own layout choice (direct, cached or
// shared kernels, cuckoo_bench.cu:822-901), scratch sizing, micro-launches,
// synchronous failure read-back after each launch and journal commits.  The
// only departure from a `cuckoo_bench` run is that Params.buckets and
// Params.kick may be overridden (the reference CLI derives both from PNUM,
// cuckoo_bench.cu:500-512), with the derived fields recomputed by the
// reference formula (cuckoo_bench.cu:513-525), as oracle/ref_harness.cpp does
// for the CPU path.
#define main reference_cuckoo_bench_main
#include "cuckoo_bench.cu"
#undef main

namespace {

Params ref_gpu_params(const Options& o, uint32_t buckets_override, uint32_t kick_override) {
    Params p = parameters(o);
    if (kick_override) p.kick = kick_override;
    if (buckets_override) {
        p.buckets = buckets_override;
        const uint64_t source = (uint64_t(1) << o.ell_i) * 3;
        p.bucket_size = source / p.buckets + (source % p.buckets != 0);
        p.ell_d = (uint32_t)std::ceil(original_log2_u64(p.bucket_size));
        p.domain = p.buckets * p.bucket_size;
        uint32_t bits = std::max<uint32_t>(bit_width_u64(p.domain - 1), 2u);
        if (bits & 1u) ++bits;
        p.half_bits = bits / 2;
        p.mask = (1ULL << p.half_bits) - 1ULL;
    }
    return p;
}

void put(char* dst, uint32_t cap, const std::string& s) {
    if (!dst || cap == 0) return;
    const size_t n = std::min<size_t>(cap - 1, s.size());
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
}

}  // namespace

extern "C" {

// Runs batches [0, 2^(et-bt)) of the experiment (seed, parameters) through the
// reference's gpu_worker on `device`, journalling into out_dir (created; it
// must not hold a journal of other parameters), then writes the reference's
// summary.json and failures.csv there.  *out_seconds: wall time of the
// worker, the reference's work_elapsed_seconds (cuckoo_bench.cu:1100,1129).
// `layout` is the reference's --table-layout value ("auto", "global",
// "shared").  Returns 0, or -1 with the exception text in err.
int ref_gpu_run(int device, const char* mode, const char* input_mode, uint32_t pnum,
                uint32_t ell_i, uint32_t buckets_override, uint32_t kick_override, uint64_t seed,
                uint32_t et, uint32_t bt, const char* layout, const char* out_dir,
                double* out_seconds, uint64_t* out_completed, uint64_t* out_failed, char* info,
                uint32_t info_cap) {
    try {
        Options o;
        o.mode = mode;
        o.input_mode = input_mode;
        o.pnum = pnum;
        o.ell_i = ell_i;
        o.et = et;
        o.bt = bt;
        o.seed = seed;
        o.out = out_dir;
        o.workers = 1;
        o.table_layout = layout ? layout : "auto";
        o.stop_after = ~0ULL;  // never stop on the failure threshold
        const Params p = ref_gpu_params(o, buckets_override, kick_override);
        fs::create_directories(o.out);
        Counters s;
        const auto done = resume(o, p, s);
        CK(cudaSetDevice(device));
        upload_aes_tables();
        aes_self_test();
        if (round_cache_enabled(o, p)) cached_aes_self_test();
        std::mutex print_mutex;
        const auto t0 = steady_ns();
        gpu_worker(0, device, o, p, done, s, print_mutex);
        const double secs = double(steady_ns() - t0) * 1e-9;
        Counters recovered;
        resume(o, p, recovered);
        final_outputs(o, p, recovered, secs, "complete", secs);
        if (out_seconds) *out_seconds = secs;
        if (out_completed) *out_completed = recovered.completed.load();
        if (out_failed) *out_failed = recovered.failed.load();
        put(info, info_cap, std::string("layout=") + table_layout_name(o, p) +
                                " buckets=" + std::to_string(p.buckets) +
                                " kick=" + std::to_string(p.kick) +
                                " half_bits=" + std::to_string(p.half_bits));
        return 0;
    } catch (const std::exception& e) {
        put(info, info_cap, e.what());
        return -1;
    }
}

}  // extern "C"
