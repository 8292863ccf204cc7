// cuckoo_bench -- command-line front end with the reference's flags, journal
// and exports (cuckoo_bench.cu:1062-1142), running the trials through the C
// ABI of libcmc.so.  One host thread per worker, each with its own device
// context, claims batch ids from a shared counter and appends to its own
// journal; batches are independent, so workers need no communication.
#include <cuda_runtime.h>

#include <chrono>
#include <exception>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <thread>

#include "cmc.h"
#include "cmc_runner.hpp"

using namespace cmc;

namespace {

void check(int rc, cmc_ctx* ctx, const char* what) {
    if (rc != CMC_OK)
        throw std::runtime_error(std::string(what) + ": " + cmc_last_error(ctx) + " (code " +
                                 std::to_string(rc) + ")");
}

void configure(cmc_ctx* ctx, const Options& o, const cmc_params& p) {
    if (o.prp_cache == "off") check(cmc_set_option(ctx, "method", 0), ctx, "--prp-cache");
    if (o.prp_cache == "on") {
        if (p.half_bits > 12)
            throw std::runtime_error("PRP round cache requires half_bits <=12; use auto/off");
        check(cmc_set_option(ctx, "method", 1), ctx, "--prp-cache");
    }
    if (o.force_global || o.table_layout == "global")
        check(cmc_set_option(ctx, "global_slots", 1), ctx, "--table-layout");
    if (o.warps_per_block)
        check(cmc_set_option(ctx, "warps_per_group", std::min<uint32_t>(o.warps_per_block, 15)), ctx,
              "--warps-per-block");
}

void worker_main(int worker, int device, const Options& o, const cmc_params& p,
                 const std::vector<uint8_t>& done, Counters& s, std::mutex& log_mutex,
                 std::string& layout) {
    cmc_ctx* ctx = nullptr;
    check(cmc_init(device, &ctx), nullptr, "cmc_init");
    std::unique_ptr<cmc_ctx, int (*)(cmc_ctx*)> guard(ctx, cmc_destroy);
    configure(ctx, o, p);
    Journal journal(o, p, worker);
    const uint64_t nb = total_batches(o);
    const uint64_t limit = o.max_batches ? std::min<uint64_t>(o.max_batches, nb) : nb;
    std::vector<uint32_t> chunk(o.micro);
    bool logged = false;
    while (!s.stop.load(std::memory_order_relaxed)) {
        if (pause_requested(o)) {
            s.stop.store(true);
            break;
        }
        const uint64_t id = s.next_batch.fetch_add(1);
        if (id >= limit) break;
        if (done[id]) continue;
        const bool committed = process_batch(
            o, id, o.micro, s,
            [&](uint32_t n, uint32_t offset, const uint32_t* key, std::vector<uint32_t>& failures) {
                uint32_t nf = 0;
                check(cmc_launch(ctx, &p, key, offset, n, chunk.data(), &nf), ctx, "cmc_launch");
                if (nf > n) throw std::runtime_error("GPU failure count out of range");
                failures.insert(failures.end(), chunk.begin(), chunk.begin() + nf);
                if (!logged) {
                    logged = true;
                    std::lock_guard<std::mutex> lock(log_mutex);
                    layout = cmc_last_plan(ctx);
                    std::cerr << "Worker " << worker << " GPU " << device << " bins=" << p.buckets
                              << " micro=" << o.micro << " " << layout << "\n";
                }
            },
            [&](uint64_t batch, uint32_t tried, const std::vector<uint32_t>& failures) {
                journal.append(batch, tried, failures);
            });
        if (!committed) break;
    }
}

void progress(const Options& o, const Counters& s, std::chrono::steady_clock::time_point start) {
    const uint64_t initial = s.completed.load(), total = 1ULL << o.et;
    while (s.active.load() > 0) {
        std::this_thread::sleep_for(std::chrono::milliseconds(200));
        static int tick = 0;
        if (++tick % 5 && s.active.load() > 0) continue;
        const uint64_t done = s.completed.load(), fail = s.failed.load();
        const double elapsed =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        const double rate = double(done - initial) / std::max(elapsed, 1e-6);
        const double eta = rate > 0 ? double(total - done) / rate : -1.0;
        const unsigned filled = unsigned(std::min<uint64_t>(30, done * 30 / total));
        std::cerr << '\r' << '[' << std::string(filled, '#') << std::string(30 - filled, '-') << "] "
                  << std::fixed << std::setprecision(2) << 100.0 * double(done) / double(total)
                  << "% | " << done << "/" << total << " | Fail " << fail << " | "
                  << std::setprecision(0) << rate << " avg exp/s | elapsed " << std::setprecision(1)
                  << elapsed << "s | ETA "
                  << (eta >= 0 ? std::to_string(uint64_t(eta)) + "s" : std::string("--")) << "     "
                  << std::flush;
    }
    std::cerr << '\n';
}

}  // namespace

int main(int argc, char** argv) {
    try {
        bool help = false;
        Options o = parse_options(argc, argv, &help);
        if (help) {
            std::cout << usage();
            return 0;
        }
        const cmc_params p = derive(o);
        fs::create_directories(o.out);
        RunLock lock(o.out);
        PauseSignals signals;
        Counters s;
        const std::vector<uint8_t> done = resume(o, p, s);
        const uint64_t planned = 1ULL << o.et;
        const uint64_t limit_batches =
            o.max_batches ? std::min<uint64_t>(o.max_batches, total_batches(o)) : total_batches(o);
        const auto start = std::chrono::steady_clock::now();
        std::cout << "mode=" << o.mode << " ET=" << o.et << " BT=" << o.bt << " PNUM=" << o.pnum
                  << " buckets=" << p.buckets << " kick=" << p.kick
                  << " bucket_size=" << p.bucket_size << " half_bits=" << p.half_bits
                  << " input_mode=" << o.input_mode << (o.k != 3 ? " k=" + std::to_string(o.k) : "")
                  << "\nResume: " << s.completed << " completed / " << s.failed << " failed\n";
        auto prefix_done = [&]() {
            for (uint64_t i = 0; i < limit_batches; ++i)
                if (!done[i]) return false;
            return true;
        };
        std::string layout = "engine=group";
        if (o.status_only || s.completed.load() == planned || pause_requested(o) ||
            s.failed.load() > o.stop_after || (o.max_batches && prefix_done())) {
            const std::string status = s.completed.load() == planned ? "complete"
                                       : pause_requested(o)          ? "paused"
                                       : s.failed.load() > o.stop_after ? "threshold"
                                       : (o.max_batches && prefix_done()) ? "budget"
                                                                          : "ready";
            final_outputs(o, p, s, 0, status, 0, layout);
            std::cout << "Status: " << status
                      << "; pending batches=" << (total_batches(o) - s.batches.load()) << "\n";
            return 0;
        }
        int gpus = 0;
        if (cudaGetDeviceCount(&gpus) != cudaSuccess || gpus == 0)
            throw std::runtime_error("No NVIDIA CUDA GPUs");
        if (o.workers == 0) o.workers = gpus;
        if (o.workers < 1 || o.workers > 256) throw std::runtime_error("workers must be in 1..256");
        if (o.workers > gpus) std::cerr << "WARNING: Multiple workers share GPUs; usually use one per GPU.\n";
        std::mutex log_mutex;
        std::vector<std::thread> threads;
        std::vector<std::exception_ptr> errors(o.workers);
        const int64_t work_start = steady_ns();
        for (int w = 0; w < o.workers; ++w) {
            s.active.fetch_add(1);
            threads.emplace_back([&, w]() {
                try {
                    worker_main(w, w % gpus, o, p, done, s, log_mutex, layout);
                } catch (...) {
                    errors[w] = std::current_exception();
                    s.abort_inflight.store(true);
                    s.stop.store(true);
                }
                mark_finished(s);
                s.active.fetch_sub(1);
            });
        }
        progress(o, s, start);
        for (auto& t : threads) t.join();
        // the journals, not the live counters, are authoritative
        Counters recovered;
        const std::vector<uint8_t> after = resume(o, p, recovered);
        bool all_prefix = true;
        for (uint64_t i = 0; i < limit_batches; ++i) all_prefix = all_prefix && after[i];
        bool error = false;
        for (auto& e : errors) error = error || bool(e);
        const std::string status = error                                ? "error"
                                   : recovered.completed.load() == planned ? "complete"
                                   : pause_requested(o)                   ? "paused"
                                   : (o.max_batches && all_prefix)        ? "budget"
                                                                          : "threshold";
        const double elapsed =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
        const double work = std::max<int64_t>(0, s.finished_ns.load() - work_start) * 1e-9;
        final_outputs(o, p, recovered, elapsed, status, work, layout);
        std::cout << "RESULT status=" << status << " completed=" << recovered.completed
                  << " failed=" << recovered.failed << " elapsed_s=" << elapsed << "\n";
        if (pause_requested(o))
            std::cout << "Paused: unfinished batches were not counted. Restart the same command to "
                         "resume. If using the PAUSE file, remove it first.\n";
        for (auto& e : errors)
            if (e) std::rethrow_exception(e);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "FATAL: " << e.what() << "\n";
        return 1;
    }
}
