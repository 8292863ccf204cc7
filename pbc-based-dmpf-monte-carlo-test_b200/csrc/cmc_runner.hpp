// cmc_runner.hpp -- host controller around the Launch seam: CLI options,
// v3 journal (checkpoint) format, resume, batch processing, exports.
//
// Behaviour and byte formats follow the reference host code
// (cuckoo_bench.cu:406-800, checkpoint.hpp) so that an existing output
// directory resumes under this runner and vice versa:
//   * journal worker_<n>.bin = 56-byte FileHeader, then per committed batch
//     RecordHeader{u64 batch, u32 tried, u32 failed}, sorted offsets,
//     RecordFooter{u32 check, u32 "END3"}; check = FNV-1a-style fold of
//     batch_lo, batch_hi, tried, count, offsets (cuckoo_bench.cu:567-581);
//   * a torn tail is cut back to the last complete record, a complete but
//     corrupt record is an error and the file is kept (cuckoo_bench.cu:650-698);
//   * a batch is committed durably (fsync) before counters move
//     (cuckoo_bench.cu:737-744).
// Additive extensions: --k (copies, 2..4), --buckets, --max-kicks.  With k = 3
// the header is the reference's version 3 byte for byte; k != 3 writes
// version 4, which appends {u32 k, u32 reserved}.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <vector>

#include "cmc.h"

namespace cmc {

namespace fs = std::filesystem;

constexpr uint32_t kJournalMagic = 0x43554b33u;  // "CUK3"
constexpr uint32_t kRecordMagic = 0x454e4433u;   // "END3"

struct Options {
    uint32_t et = 30, bt = 20, pnum = 16, ell_i = 32, micro = 1u << 17;
    uint64_t seed = 1, stop_after = 1ULL << 20;
    std::string mode = "drrt18", out = "cuckoo_results", input_mode = "sequential";
    int workers = 0;
    uint32_t scratch_mib = 256, block_threads = 256, warps_per_block = 0;
    std::string prp_cache = "auto", table_layout = "auto", shared_variant = "auto";
    std::string backend = "cuda";
    bool force_global = false, status_only = false;
    // extensions (0 = reference derivation)
    uint32_t k = 3, buckets = 0, max_kicks = 0;
    uint64_t max_batches = 0;  // run only the first N batches (trial budgets)
};

std::string usage();
// Parses argv like cuckoo_bench.cu:431-480; throws std::runtime_error with the
// reference's messages.  Sets *help when --help/-h was given.
Options parse_options(int argc, char** argv, bool* help);
cmc_params derive(const Options& o);  // throws on invalid parameters

#pragma pack(push, 1)
struct FileHeader {
    uint32_t magic = kJournalMagic, version = 3;
    uint64_t seed = 0, planned = 0;
    uint32_t et = 0, bt = 0, pnum = 0, ell_i = 0, mode = 0, buckets = 0, kick = 0, input_mode = 0;
};
struct FileHeaderExt {  // version 4 tail (k != 3)
    uint32_t k = 3, reserved = 0;
};
struct RecordHeader {
    uint64_t batch;
    uint32_t tried, failed;
};
struct RecordFooter {
    uint32_t check, magic;
};
#pragma pack(pop)
static_assert(sizeof(FileHeader) == 56, "v3 header is 56 bytes");
static_assert(sizeof(RecordHeader) == 16 && sizeof(RecordFooter) == 8, "record layout");

uint32_t record_check(uint64_t batch, uint32_t tried, const std::vector<uint32_t>& offsets);
uint64_t batch_length(const Options& o, uint64_t id);
uint64_t total_batches(const Options& o);
FileHeader make_header(const Options& o, const cmc_params& p);
size_t header_bytes(const Options& o);
std::string journal_path(const Options& o, int worker);
std::vector<std::string> journal_paths(const Options& o);

struct Counters {
    std::atomic<uint64_t> completed{0}, failed{0}, batches{0};
    std::atomic<bool> stop{false}, abort_inflight{false};
    std::atomic<int> active{0};
    std::atomic<uint64_t> next_batch{0};
    std::atomic<int64_t> finished_ns{0};
};

int64_t steady_ns();
void mark_finished(Counters& s);

// Validates every journal in o.out against the expected header, repairs torn
// tails, accumulates counters and returns the per-batch done map.
std::vector<uint8_t> resume(const Options& o, const cmc_params& p, Counters& s);

// Append-only journal of one worker.
class Journal {
   public:
    Journal(const Options& o, const cmc_params& p, int worker);
    ~Journal();
    Journal(const Journal&) = delete;
    Journal& operator=(const Journal&) = delete;
    void append(uint64_t batch, uint32_t tried, const std::vector<uint32_t>& offsets);
    FILE* file() const { return f_; }

   private:
    FILE* f_ = nullptr;
};

void durable_flush(FILE* f);

// SIGINT/SIGTERM set a flag; a PAUSE file in the output directory does too.
extern std::atomic<bool> g_pause_signal;
class PauseSignals {
   public:
    PauseSignals();
    ~PauseSignals();
    PauseSignals(const PauseSignals&) = delete;

   private:
    void (*old_int_)(int);
    void (*old_term_)(int);
};
bool pause_requested(const Options& o);

// Exclusive advisory lock on <dir>/.run.lock, released by the OS on exit.
class RunLock {
   public:
    explicit RunLock(const fs::path& dir);
    ~RunLock();
    RunLock(const RunLock&) = delete;

   private:
    int fd_ = -1;
};

// One batch through micro-launches (cuckoo_bench.cu:724-745): launch(n,
// offset, key, failures) appends failing offsets; the sorted list is committed
// before counters change; a pause or another worker's abort discards it.
template <class Launch, class Commit>
bool process_batch(const Options& o, uint64_t id, uint32_t micro, Counters& s, Launch&& launch,
                   Commit&& commit) {
    if (micro == 0) throw std::runtime_error("micro must be positive");
    uint32_t key[44];
    cmc_batch_key(o.seed, id, key);
    const uint32_t actual = static_cast<uint32_t>(batch_length(o, id));
    std::vector<uint32_t> failures;
    for (uint32_t offset = 0; offset < actual;) {
        if (s.abort_inflight.load() || pause_requested(o)) {
            s.stop.store(true);
            return false;
        }
        const uint32_t n = std::min<uint32_t>(micro, actual - offset);
        launch(n, offset, key, failures);
        offset += n;
    }
    std::sort(failures.begin(), failures.end());
    commit(id, actual, failures);
    s.completed.fetch_add(actual, std::memory_order_relaxed);
    const uint64_t total = s.failed.fetch_add(failures.size()) + failures.size();
    s.batches.fetch_add(1);
    if (total > o.stop_after) s.stop.store(true);
    return true;
}

// summary.json and failures.csv (cuckoo_bench.cu:746-800).
void final_outputs(const Options& o, const cmc_params& p, const Counters& s, double seconds,
                   const std::string& status, double work_seconds, const std::string& layout);

}  // namespace cmc
