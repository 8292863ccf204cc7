// cmc_runner.cpp -- host controller: options, journal, resume, exports.
#include "cmc_runner.hpp"

#include <fcntl.h>
#include <sys/file.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <csignal>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <memory>
#include <stdexcept>

namespace cmc {

std::atomic<bool> g_pause_signal{false};

namespace {

uint64_t parse_u64(const std::string& s) {
    if (s.empty() || s[0] == '-') throw std::runtime_error("Invalid unsigned number: " + s);
    size_t at = 0;
    unsigned long long v = 0;
    try {
        v = std::stoull(s, &at, 0);
    } catch (const std::exception&) {
        throw std::runtime_error("Invalid number: " + s);
    }
    if (at != s.size()) throw std::runtime_error("Invalid number: " + s);
    return v;
}

uint32_t parse_u32(const std::string& s) {
    const uint64_t v = parse_u64(s);
    if (v > std::numeric_limits<uint32_t>::max()) throw std::runtime_error("Number exceeds uint32: " + s);
    return static_cast<uint32_t>(v);
}

void on_pause_signal(int) { g_pause_signal.store(true, std::memory_order_relaxed); }

}  // namespace

std::string usage() {
    return "Usage: ./cuckoo_bench --mode bgh25|drrt18 --et 40 --bt 20 "
           "--pnum 16 --seed 123 --workers 1 --micro 131072 "
           "--out results [--input-mode sequential|affine] "
           "[--scratch-mib 256] [--prp-cache auto|on|off] [--block-threads 256] "
           "[--table-layout auto|global|shared] [--shared-variant auto|round|map] "
           "[--warps-per-block N] [--stop-after 1048576] [--global-table] [--status] "
           "[--k 3] [--buckets B] [--max-kicks K] [--max-batches N]\n";
}

Options parse_options(int argc, char** argv, bool* help) {
    Options o;
    if (help) *help = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--help" || a == "-h") {
            if (help) *help = true;
            return o;
        }
        if (a == "--global-table") { o.force_global = true; continue; }
        if (a == "--status") { o.status_only = true; continue; }
        if (i + 1 >= argc) throw std::runtime_error("Missing value after " + a);
        const std::string v = argv[++i];
        if (a == "--et") o.et = parse_u32(v);
        else if (a == "--bt") o.bt = parse_u32(v);
        else if (a == "--pnum") o.pnum = parse_u32(v);
        else if (a == "--ell-i") o.ell_i = parse_u32(v);
        else if (a == "--micro") o.micro = parse_u32(v);
        else if (a == "--scratch-mib") o.scratch_mib = parse_u32(v);
        else if (a == "--prp-cache") o.prp_cache = v;
        else if (a == "--block-threads") o.block_threads = parse_u32(v);
        else if (a == "--table-layout") o.table_layout = v;
        else if (a == "--shared-variant") o.shared_variant = v;
        else if (a == "--warps-per-block") o.warps_per_block = parse_u32(v);
        else if (a == "--seed") o.seed = parse_u64(v);
        else if (a == "--workers") {
            const uint64_t n = parse_u64(v);
            if (n > 256) throw std::runtime_error("workers exceeds 256");
            o.workers = static_cast<int>(n);
        } else if (a == "--stop-after") o.stop_after = parse_u64(v);
        else if (a == "--mode") o.mode = v;
        else if (a == "--input-mode") o.input_mode = v;
        else if (a == "--out") o.out = v;
        else if (a == "--k") o.k = parse_u32(v);
        else if (a == "--buckets") o.buckets = parse_u32(v);
        else if (a == "--max-kicks") o.max_kicks = parse_u32(v);
        else if (a == "--max-batches") o.max_batches = parse_u64(v);
        else throw std::runtime_error("Unknown option " + a);
    }
    // the reference's bounds (cuckoo_bench.cu:467-478), plus k in 2..4
    if (o.et > 40 || o.bt > 30 || o.bt > o.et || o.et == 0 || o.bt == 0 || o.pnum < 3 ||
        o.pnum > 65534 || o.micro == 0 || o.scratch_mib == 0 || o.ell_i > 61 ||
        (o.block_threads != 64 && o.block_threads != 128 && o.block_threads != 256) ||
        (o.prp_cache != "auto" && o.prp_cache != "on" && o.prp_cache != "off") ||
        (o.table_layout != "auto" && o.table_layout != "global" && o.table_layout != "shared") ||
        (o.shared_variant != "auto" && o.shared_variant != "round" && o.shared_variant != "map") ||
        o.warps_per_block > 32 || (o.ell_i < 16 && (1ULL << o.ell_i) < o.pnum) ||
        (o.mode != "bgh25" && o.mode != "drrt18") ||
        (o.input_mode != "sequential" && o.input_mode != "affine") || o.k < 2 || o.k > 4)
        throw std::runtime_error(
            "Invalid config (ET 1..40, BT 1..min(ET,30), PNUM 3..65534, ell-i <=61, "
            "2^ell-i >=PNUM, input mode sequential|affine)");
    if (o.table_layout == "shared" && o.force_global)
        throw std::runtime_error("--table-layout shared conflicts with --global-table");
    return o;
}

cmc_params derive(const Options& o) {
    cmc_params p{};
    const int rc = cmc_derive_params(o.mode == "bgh25" ? CMC_MODE_BGH25 : CMC_MODE_DRRT18, o.pnum,
                                     o.ell_i, o.k, o.buckets, o.max_kicks,
                                     o.input_mode == "sequential" ? CMC_INPUT_SEQUENTIAL
                                                                  : CMC_INPUT_AFFINE,
                                     &p);
    if (rc) throw std::runtime_error("Invalid experiment parameters (PRP domain overflow or k/B out of range)");
    return p;
}

uint32_t record_check(uint64_t batch, uint32_t tried, const std::vector<uint32_t>& offsets) {
    uint32_t h = 0x811c9dc5u;
    auto fold = [&h](uint32_t x) { h = (h ^ x) * 0x01000193u; };
    fold(static_cast<uint32_t>(batch));
    fold(static_cast<uint32_t>(batch >> 32));
    fold(tried);
    fold(static_cast<uint32_t>(offsets.size()));
    for (uint32_t x : offsets) fold(x);
    return h;
}

uint64_t total_batches(const Options& o) { return 1ULL << (o.et - o.bt); }

uint64_t batch_length(const Options& o, uint64_t id) {
    const uint64_t total = 1ULL << o.et, start = id << o.bt;
    return std::min<uint64_t>(1ULL << o.bt, total - start);
}

FileHeader make_header(const Options& o, const cmc_params& p) {
    FileHeader h;
    h.version = o.k == 3 ? 3 : 4;
    h.seed = o.seed;
    h.planned = 1ULL << o.et;
    h.et = o.et;
    h.bt = o.bt;
    h.pnum = o.pnum;
    h.ell_i = o.ell_i;
    h.mode = o.mode == "bgh25" ? 1 : 2;
    h.buckets = p.buckets;
    h.kick = p.kick;
    h.input_mode = o.input_mode == "sequential" ? 0 : 1;
    return h;
}

size_t header_bytes(const Options& o) {
    return sizeof(FileHeader) + (o.k == 3 ? 0 : sizeof(FileHeaderExt));
}

std::string journal_path(const Options& o, int worker) {
    return o.out + "/worker_" + std::to_string(worker) + ".bin";
}

std::vector<std::string> journal_paths(const Options& o) {
    std::vector<std::string> paths;
    for (const auto& e : fs::directory_iterator(o.out)) {
        if (!e.is_regular_file()) continue;
        const std::string name = e.path().filename().string();
        if (name.size() < 12 || name.rfind("worker_", 0) != 0 ||
            name.compare(name.size() - 4, 4, ".bin") != 0)
            continue;
        const std::string digits = name.substr(7, name.size() - 11);
        if (digits.empty() ||
            !std::all_of(digits.begin(), digits.end(), [](char c) { return c >= '0' && c <= '9'; }))
            continue;
        paths.push_back(e.path().string());
    }
    std::sort(paths.begin(), paths.end());
    return paths;
}

int64_t steady_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

void mark_finished(Counters& s) {
    const int64_t now = steady_ns();
    int64_t prev = s.finished_ns.load();
    while (prev < now && !s.finished_ns.compare_exchange_weak(prev, now)) {
    }
}

namespace {

bool same_header(const FileHeader& a, const FileHeader& b) {
    return a.magic == b.magic && a.version == b.version && a.seed == b.seed &&
           a.planned == b.planned && a.et == b.et && a.bt == b.bt && a.pnum == b.pnum &&
           a.ell_i == b.ell_i && a.mode == b.mode && a.buckets == b.buckets && a.kick == b.kick &&
           a.input_mode == b.input_mode;
}

bool sorted_unique_below(const std::vector<uint32_t>& v, uint32_t limit) {
    for (size_t i = 1; i < v.size(); ++i)
        if (v[i] <= v[i - 1]) return false;
    return v.empty() || v.back() < limit;
}

}  // namespace

std::vector<uint8_t> resume(const Options& o, const cmc_params& p, Counters& s) {
    const uint64_t nb = total_batches(o);
    if (nb > (1ULL << 28)) throw std::runtime_error("Too many batches for the completion bitmap; increase --bt");
    std::vector<uint8_t> done(static_cast<size_t>(nb), 0);
    const FileHeader want = make_header(o, p);
    const size_t hb = header_bytes(o);
    const auto paths = journal_paths(o);
    // every complete header is validated before any tail is repaired
    for (const auto& path : paths) {
        if (fs::file_size(path) < hb) continue;
        std::ifstream in(path, std::ios::binary);
        FileHeader h{};
        FileHeaderExt x{};
        in.read(reinterpret_cast<char*>(&h), sizeof h);
        if (o.k != 3) in.read(reinterpret_cast<char*>(&x), sizeof x);
        if (!in) throw std::runtime_error("Cannot read journal header: " + path);
        if (!same_header(h, want) || (o.k != 3 && x.k != o.k))
            throw std::runtime_error("Existing journal has different experiment parameters");
    }
    for (const auto& path : paths) {
        const uint64_t size = fs::file_size(path);
        if (size < hb) {
            fs::resize_file(path, 0);
            continue;
        }
        std::ifstream in(path, std::ios::binary);
        in.seekg(static_cast<std::streamoff>(hb));
        uint64_t safe = hb;
        while (safe < size) {
            if (size - safe < sizeof(RecordHeader)) break;  // torn record header
            RecordHeader r{};
            in.read(reinterpret_cast<char*>(&r), sizeof r);
            if (!in) throw std::runtime_error("Journal read failed: " + path);
            if (r.batch >= nb || r.tried != batch_length(o, r.batch) || r.failed > r.tried)
                throw std::runtime_error("Invalid journal record header: " + path);
            const uint64_t bytes = sizeof r + uint64_t(r.failed) * 4 + sizeof(RecordFooter);
            if (size - safe < bytes) break;  // uncommitted partial tail
            std::vector<uint32_t> offsets(r.failed);
            if (r.failed) in.read(reinterpret_cast<char*>(offsets.data()), std::streamsize(r.failed) * 4);
            RecordFooter f{};
            in.read(reinterpret_cast<char*>(&f), sizeof f);
            if (!in) throw std::runtime_error("Journal read failed: " + path);
            if (f.magic != kRecordMagic || f.check != record_check(r.batch, r.tried, offsets))
                throw std::runtime_error("Corrupt complete journal record (file preserved): " + path);
            if (!sorted_unique_below(offsets, r.tried))
                throw std::runtime_error("Invalid journal offsets: " + path);
            if (done[r.batch]) throw std::runtime_error("Duplicate committed batch: " + std::to_string(r.batch));
            done[r.batch] = 1;
            s.batches.fetch_add(1);
            s.completed.fetch_add(r.tried);
            s.failed.fetch_add(r.failed);
            safe += bytes;
        }
        in.close();
        if (size != safe) fs::resize_file(path, safe);
    }
    return done;
}

void durable_flush(FILE* f) {
    if (std::fflush(f) != 0) throw std::runtime_error("Journal flush failed");
    if (::fsync(::fileno(f)) != 0) throw std::runtime_error("Journal disk sync failed");
}

Journal::Journal(const Options& o, const cmc_params& p, int worker) {
    const std::string path = journal_path(o, worker);
    const bool existing = fs::exists(path) && fs::file_size(path) != 0;
    f_ = std::fopen(path.c_str(), existing ? "ab" : "wb");
    if (!f_) throw std::runtime_error("Unable to open: " + path);
    if (!existing) {
        const FileHeader h = make_header(o, p);
        bool ok = std::fwrite(&h, sizeof h, 1, f_) == 1;
        if (ok && o.k != 3) {
            FileHeaderExt x;
            x.k = o.k;
            ok = std::fwrite(&x, sizeof x, 1, f_) == 1;
        }
        if (!ok) {
            std::fclose(f_);
            f_ = nullptr;
            throw std::runtime_error("Journal header write failed");
        }
        durable_flush(f_);
    }
}

Journal::~Journal() {
    if (f_) std::fclose(f_);
}

void Journal::append(uint64_t batch, uint32_t tried, const std::vector<uint32_t>& offsets) {
    if (offsets.size() > tried) throw std::runtime_error("Invalid failure count");
    if (!sorted_unique_below(offsets, tried)) throw std::runtime_error("Invalid failure offsets");
    const RecordHeader h{batch, tried, static_cast<uint32_t>(offsets.size())};
    const RecordFooter f{record_check(batch, tried, offsets), kRecordMagic};
    if (std::fwrite(&h, sizeof h, 1, f_) != 1 ||
        (!offsets.empty() && std::fwrite(offsets.data(), 4, offsets.size(), f_) != offsets.size()) ||
        std::fwrite(&f, sizeof f, 1, f_) != 1)
        throw std::runtime_error("Journal write failed");
    durable_flush(f_);
}

PauseSignals::PauseSignals() {
    g_pause_signal.store(false);
    old_int_ = std::signal(SIGINT, on_pause_signal);
    if (old_int_ == SIG_ERR) throw std::runtime_error("Cannot install SIGINT handler");
    old_term_ = std::signal(SIGTERM, on_pause_signal);
    if (old_term_ == SIG_ERR) {
        std::signal(SIGINT, old_int_);
        throw std::runtime_error("Cannot install SIGTERM handler");
    }
}

PauseSignals::~PauseSignals() {
    std::signal(SIGINT, old_int_);
    std::signal(SIGTERM, old_term_);
}

bool pause_requested(const Options& o) {
    return g_pause_signal.load(std::memory_order_relaxed) || fs::exists(fs::path(o.out) / "PAUSE");
}

RunLock::RunLock(const fs::path& dir) {
    const std::string path = (dir / ".run.lock").string();
    fd_ = ::open(path.c_str(), O_CREAT | O_RDWR, 0600);
    if (fd_ < 0) throw std::runtime_error("Cannot open run lock: " + path);
    if (::flock(fd_, LOCK_EX | LOCK_NB) != 0) {
        ::close(fd_);
        fd_ = -1;
        throw std::runtime_error("Another process is using the output directory: " + path);
    }
}

RunLock::~RunLock() {
    if (fd_ >= 0) {
        ::flock(fd_, LOCK_UN);
        ::close(fd_);
    }
}

void final_outputs(const Options& o, const cmc_params& p, const Counters& s, double seconds,
                   const std::string& status, double work_seconds, const std::string& layout) {
    const uint64_t completed = s.completed.load(), fails = s.failed.load(), batches = s.batches.load();
    {
        std::ofstream out;
        out.exceptions(std::ios::failbit | std::ios::badbit);
        out.open(o.out + "/summary.json", std::ios::trunc);
        const bool cache = o.prp_cache != "off" && p.half_bits <= 12;
        out << "{\n  \"status\": \"" << status << "\",\n  \"seed_scheme\": \"aes-batch-v1\",\n"
            << "  \"mode\": \"" << o.mode << "\",\n  \"algorithm\": \"prp-cuckoo-aes-feistel-port\",\n"
            << "  \"backend\": \"" << o.backend << "\",\n  \"workers\": " << o.workers << ",\n"
            << "  \"micro_requested\": " << o.micro << ",\n  \"scratch_mib\": " << o.scratch_mib << ",\n"
            << "  \"prp_cache_requested\": \"" << o.prp_cache << "\",\n"
            << "  \"prp_cache_enabled\": " << (cache ? "true" : "false") << ",\n"
            << "  \"table_layout_requested\": \"" << o.table_layout << "\",\n"
            << "  \"table_layout_planned\": \"" << layout << "\",\n"
            << "  \"shared_variant_requested\": \"" << o.shared_variant << "\",\n"
            << "  \"block_threads_requested\": " << o.block_threads << ",\n"
            << "  \"warps_per_block_requested\": " << o.warps_per_block << ",\n"
            << "  \"input_mode\": \"" << o.input_mode << "\",\n"
            << "  \"seed\": " << o.seed << ",\n  \"ET\": " << o.et << ",\n  \"BT\": " << o.bt << ",\n"
            << "  \"seed_decimal\": \"" << o.seed << "\",\n  \"batch_size\": " << (1ULL << o.bt) << ",\n"
            << "  \"PNUM_T\": " << o.pnum << ",\n  \"ELL_I\": " << o.ell_i << ",\n";
        if (o.k != 3) out << "  \"K_COPIES\": " << o.k << ",\n";
        out << "  \"BUCKETS_NUM\": " << p.buckets << ",\n  \"MAX_KICK_TIMES\": " << p.kick << ",\n"
            << "  \"BUCKET_SIZE\": " << p.bucket_size << ",\n  \"PRP_DOMAIN\": " << p.domain << ",\n"
            << "  \"planned\": " << (1ULL << o.et) << ",\n  \"completed\": " << completed
            << ",\n  \"failed\": " << fails << ",\n  \"completed_batches\": " << batches
            << ",\n  \"pending_batches\": " << (total_batches(o) - batches)
            << ",\n  \"failed_ratio\": " << std::setprecision(17)
            << (completed ? double(fails) / double(completed) : 0.0)
            << ",\n  \"elapsed_seconds\": " << seconds
            << ",\n  \"work_elapsed_seconds\": " << work_seconds << ",\n  \"threshold_exceeded\": "
            << (fails > o.stop_after ? "true" : "false") << "\n}\n";
    }
    std::ofstream csv;
    csv.exceptions(std::ios::failbit | std::ios::badbit);
    csv.open(o.out + "/failures.csv", std::ios::trunc);
    csv << "batch_id,offset\n";
    uint64_t count = 0;
    const size_t hb = header_bytes(o);
    for (const auto& path : journal_paths(o)) {
        std::ifstream in(path, std::ios::binary);
        if (!in) continue;
        in.seekg(static_cast<std::streamoff>(hb), std::ios::beg);
        for (;;) {
            RecordHeader r{};
            in.read(reinterpret_cast<char*>(&r), sizeof r);
            if (!in) break;
            for (uint32_t i = 0; i < r.failed; ++i) {
                uint32_t off = 0;
                in.read(reinterpret_cast<char*>(&off), sizeof off);
                csv << r.batch << ',' << off << '\n';
                ++count;
            }
            in.seekg(sizeof(RecordFooter), std::ios::cur);
            if (!in) throw std::runtime_error("Corrupt journal in final export");
        }
    }
    if (count != fails) throw std::runtime_error("Exported failure count mismatch");
}

}  // namespace cmc
