// host_tests -- controller, journal and resume tests without a GPU.
// Scenarios follow the reference's host_tests.cpp (mock launcher,
// pause/abort, torn tails, corrupt records, duplicates, parameter changes,
// lock, argument bounds); the launcher here is a deterministic mock that also
// checks the batch key handed to it.
#include <array>
#include <csignal>
#include <cstring>
#include <fstream>
#include <iostream>
#include <set>
#include <thread>

#include "cmc.h"
#include "cmc_grants.hpp"
#include "cmc_runner.hpp"

using namespace cmc;

namespace {

int g_checks = 0;

void require(bool ok, const char* what) {
    ++g_checks;
    if (!ok) throw std::runtime_error(what);
}

template <class F>
void must_throw(F f, const char* what) {
    bool threw = false;
    try {
        f();
    } catch (const std::exception&) {
        threw = true;
    }
    require(threw, what);
}

void mock_launch(uint64_t id, uint32_t n, uint32_t offset, const uint32_t* key,
                 std::vector<uint32_t>& failures) {
    uint32_t want[44];
    cmc_batch_key(123, id, want);
    require(std::memcmp(key, want, sizeof want) == 0, "batch key changed with scheduling");
    for (uint32_t j = offset; j < offset + n; ++j)
        if ((id * 8 + j) % 7 == 0) failures.push_back(j);
}

bool run_batch(const Options& o, uint64_t id, uint32_t micro, Counters& s, Journal& j) {
    return process_batch(
        o, id, micro, s,
        [&](uint32_t n, uint32_t off, const uint32_t* key, std::vector<uint32_t>& f) {
            mock_launch(id, n, off, key, f);
        },
        [&](uint64_t b, uint32_t n, const std::vector<uint32_t>& f) { j.append(b, n, f); });
}

Options make_options(const fs::path& root, const char* name) {
    Options o;
    o.et = 6;
    o.bt = 3;
    o.seed = 123;
    o.pnum = 16;
    o.ell_i = 8;
    o.out = (root / name).string();
    fs::create_directories(o.out);
    return o;
}

std::set<std::string> csv_rows(const Options& o) {
    std::ifstream f(fs::path(o.out) / "failures.csv");
    std::string line;
    std::getline(f, line);
    std::set<std::string> rows;
    while (std::getline(f, line)) rows.insert(line);
    return rows;
}

void check_keys() {
    const uint32_t expected[2][4] = {{0x992dc0b2, 0xecc207f0, 0x5f9a7017, 0x1fb84a2f},
                                     {0x58f85b99, 0xfc3cbd02, 0x022bf19c, 0x10dad53d}};
    const uint64_t ids[2] = {0, 7};
    for (int i = 0; i < 2; ++i) {
        uint32_t key[44], out[4];
        const uint32_t zero[4] = {0, 0, 0, 0};
        cmc_batch_key(123, ids[i], key);
        cmc_host_aes128(key, zero, out);
        require(std::memcmp(out, expected[i], sizeof out) == 0, "batch-key vector changed");
    }
}

void check_pause(const fs::path& root) {
    {
        auto o = make_options(root, "pause");
        const auto p = derive(o);
        Counters s;
        PauseSignals signals;
        unsigned launches = 0;
        {
            Journal j(o, p, 0);
            const bool r = process_batch(
                o, 0, 2, s,
                [&](uint32_t n, uint32_t off, const uint32_t* key, std::vector<uint32_t>& f) {
                    mock_launch(0, n, off, key, f);
                    ++launches;
                    std::raise(SIGINT);
                },
                [&](uint64_t b, uint32_t n, const std::vector<uint32_t>& f) { j.append(b, n, f); });
            require(!r && launches == 1 && s.completed == 0 && s.failed == 0, "partial batch was counted");
        }
        Counters r;
        auto done = resume(o, p, r);
        require(!done[0] && r.completed == 0, "partial batch was persisted");
        g_pause_signal.store(false);
        s.stop.store(false);
        {
            Journal j(o, p, 0);
            require(run_batch(o, 0, 3, s, j), "unfinished batch did not restart");
        }
        require(s.completed == 8 && s.failed == 2, "restart counts wrong");
        Counters saved;
        done = resume(o, p, saved);
        require(done[0] && saved.completed == 8, "completed batch not recovered");
    }
    {
        auto o = make_options(root, "pause_after_last_micro");
        const auto p = derive(o);
        Counters s;
        Journal j(o, p, 0);
        const bool r = process_batch(
            o, 0, 8, s,
            [&](uint32_t n, uint32_t off, const uint32_t* key, std::vector<uint32_t>& f) {
                mock_launch(0, n, off, key, f);
                g_pause_signal.store(true);
            },
            [&](uint64_t b, uint32_t n, const std::vector<uint32_t>& f) { j.append(b, n, f); });
        require(r && s.completed == 8, "fully finished batch was discarded on pause");
        g_pause_signal.store(false);
    }
    {
        auto o = make_options(root, "pause_file");
        const auto p = derive(o);
        std::ofstream(fs::path(o.out) / "PAUSE").close();
        Counters s;
        Journal j(o, p, 0);
        require(!run_batch(o, 0, 2, s, j) && s.completed == 0, "PAUSE file ignored");
        fs::remove(fs::path(o.out) / "PAUSE");
    }
    {
        auto o = make_options(root, "worker_error");
        const auto p = derive(o);
        Counters s;
        {
            Journal j(o, p, 0);
            unsigned calls = 0;
            must_throw(
                [&] {
                    process_batch(
                        o, 0, 2, s,
                        [&](uint32_t n, uint32_t off, const uint32_t* key, std::vector<uint32_t>& f) {
                            if (++calls == 2) throw std::runtime_error("mock GPU error");
                            mock_launch(0, n, off, key, f);
                        },
                        [&](uint64_t b, uint32_t n, const std::vector<uint32_t>& f) { j.append(b, n, f); });
                },
                "GPU error was ignored");
            s.abort_inflight.store(true);
            require(!run_batch(o, 1, 2, s, j), "another worker's abort was ignored");
        }
        Counters r;
        resume(o, p, r);
        require(r.completed == 0, "failed batch was committed");
    }
}

void check_journals(const fs::path& root) {
    auto o = make_options(root, "holes");
    const auto p = derive(o);
    Counters s;
    {
        Journal j(o, p, 3);
        run_batch(o, 6, 2, s, j);
        run_batch(o, 2, 2, s, j);
    }
    const auto path = journal_path(o, 3);
    const auto safe = fs::file_size(path);
    {
        std::ofstream f(path, std::ios::binary | std::ios::app);
        RecordHeader h{1, 8, 1};
        f.write(reinterpret_cast<const char*>(&h), sizeof h);
        f.write("x", 1);
    }
    Counters restored;
    auto done = resume(o, p, restored);
    require(done[6] && done[2] && !done[1] && restored.completed == 16, "out-of-order restore failed");
    require(fs::file_size(path) == safe, "torn tail was not removed");
    // finish the holes with another worker count and micro size
    std::vector<std::thread> workers;
    std::array<std::exception_ptr, 3> errors{};
    for (int w = 0; w < 3; ++w)
        workers.emplace_back([&, w] {
            try {
                Journal j(o, p, w);
                for (;;) {
                    const uint64_t id = restored.next_batch.fetch_add(1);
                    if (id >= done.size()) break;
                    if (done[id]) continue;
                    run_batch(o, id, 5, restored, j);
                }
            } catch (...) {
                errors[w] = std::current_exception();
            }
        });
    for (auto& w : workers) w.join();
    for (auto& e : errors)
        if (e) std::rethrow_exception(e);
    Counters recovered;
    done = resume(o, p, recovered);
    require(recovered.completed == 64 && recovered.batches == 8 && recovered.failed == 10,
            "resume double-counted or omitted work");
    final_outputs(o, p, recovered, 0, "complete", 0, "mock");
    auto one = make_options(root, "one_shot");
    const auto onep = derive(one);
    Counters ones;
    {
        Journal j(one, onep, 0);
        for (uint64_t id = 0; id < 8; ++id) run_batch(one, id, 1, ones, j);
    }
    final_outputs(one, onep, ones, 0, "complete", 0, "mock");
    require(csv_rows(o) == csv_rows(one), "pause/resume differs from uninterrupted run");

    auto torn = make_options(root, "torn_file_header");
    const auto tp = derive(torn);
    {
        std::ofstream f(journal_path(torn, 0), std::ios::binary);
        f.write("CUK", 3);
    }
    Counters tc;
    resume(torn, tp, tc);
    {
        Journal j(torn, tp, 0);
        require(run_batch(torn, 0, 2, tc, j), "header repair failed");
    }
    Counters tr;
    resume(torn, tp, tr);
    require(tr.completed == 8, "repaired header not usable");

    auto crash = make_options(root, "commit_before_counter_crash");
    const auto cp = derive(crash);
    Counters cs;
    {
        Journal j(crash, cp, 0);
        must_throw(
            [&] {
                process_batch(
                    crash, 0, 4, cs,
                    [&](uint32_t n, uint32_t off, const uint32_t* key, std::vector<uint32_t>& f) {
                        mock_launch(0, n, off, key, f);
                    },
                    [&](uint64_t b, uint32_t n, const std::vector<uint32_t>& f) {
                        j.append(b, n, f);
                        throw std::runtime_error("crash");
                    });
            },
            "mock crash did not throw");
    }
    require(cs.completed == 0, "mock crash published counters");
    Counters cr;
    resume(crash, cp, cr);
    require(cr.completed == 8, "durable commit lost before counter update");

    auto corrupt = make_options(root, "corrupt");
    const auto xp = derive(corrupt);
    Counters xc;
    {
        Journal j(corrupt, xp, 0);
        run_batch(corrupt, 0, 8, xc, j);
    }
    const auto xfile = journal_path(corrupt, 0);
    const auto xsize = fs::file_size(xfile);
    {
        std::fstream f(xfile, std::ios::binary | std::ios::in | std::ios::out);
        f.seekp(-1, std::ios::end);
        f.put('\0');
    }
    Counters xr;
    must_throw([&] { resume(corrupt, xp, xr); }, "corrupt complete record was accepted");
    require(fs::file_size(xfile) == xsize, "corrupt complete record was truncated");

    auto dup = make_options(root, "duplicate");
    const auto dp = derive(dup);
    Counters dc;
    {
        Journal j(dup, dp, 0);
        run_batch(dup, 0, 8, dc, j);
    }
    {
        Journal j(dup, dp, 1);
        run_batch(dup, 0, 8, dc, j);
    }
    Counters dr;
    must_throw([&] { resume(dup, dp, dr); }, "duplicate batch was accepted");
    auto different = o;
    different.seed = 124;
    Counters mismatch;
    must_throw([&] { resume(different, p, mismatch); }, "mismatched seed was accepted");
}

void check_k_extension(const fs::path& root) {
    auto o = make_options(root, "k4");
    o.k = 4;
    const auto p = derive(o);
    Counters s;
    {
        Journal j(o, p, 0);
        run_batch(o, 0, 8, s, j);
    }
    require(fs::file_size(journal_path(o, 0)) == 64 + 16 + 4 * 2 + 8, "v4 journal layout");
    Counters r;
    auto done = resume(o, p, r);
    require(done[0] && r.completed == 8, "v4 journal not resumable");
    auto three = o;
    three.k = 3;
    Counters m;
    must_throw([&] { resume(three, derive(three), m); }, "k change was accepted");
    // a k = 3 header is the reference's 56-byte version 3
    auto v3 = make_options(root, "k3");
    const auto p3 = derive(v3);
    { Journal j(v3, p3, 0); }
    require(fs::file_size(journal_path(v3, 0)) == 56, "v3 header size");
    std::ifstream in(journal_path(v3, 0), std::ios::binary);
    FileHeader h{};
    in.read(reinterpret_cast<char*>(&h), sizeof h);
    require(h.magic == 0x43554b33u && h.version == 3 && h.planned == 64 && h.buckets == 23 &&
                h.kick == 100 && h.mode == 2,
            "v3 header fields");
}

void check_locks_and_parameters(const fs::path& root) {
    auto o = make_options(root, "locks");
    {
        RunLock lock(o.out);
        must_throw([&] { RunLock another(o.out); }, "concurrent directory lock accepted");
    }
    { RunLock lock(o.out); }
    auto parse = [](std::vector<std::string> args) {
        std::vector<char*> argv;
        static std::string name = "bench";
        argv.push_back(&name[0]);
        for (auto& a : args) argv.push_back(&a[0]);
        bool help = false;
        return parse_options(int(argv.size()), argv.data(), &help);
    };
    must_throw([&] { parse({"--seed", "-1"}); }, "negative unsigned argument accepted");
    must_throw([&] { parse({"--pnum", "4294967296"}); }, "overflowing argument accepted");
    require(parse({"--scratch-mib", "2048"}).scratch_mib == 2048, "GPU budget argument ignored");
    must_throw([&] { parse({"--scratch-mib", "0"}); }, "zero GPU budget accepted");
    must_throw([&] { parse({"--bt", "7", "--et", "6"}); }, "BT > ET accepted");
    must_throw([&] { parse({"--k", "5"}); }, "k = 5 accepted");
    must_throw([&] { parse({"--frobnicate", "1"}); }, "unknown option accepted");
    require(parse({"--mode", "bgh25", "--buckets", "96", "--max-kicks", "100"}).buckets == 96,
            "--buckets ignored");
    auto p = derive(o);
    require(p.buckets == 23, "DRRT18 parameter derivation changed");
    o.mode = "bgh25";
    require(derive(o).buckets == 32, "BGH25 parameter derivation changed");
}

}  // namespace

// The serving grant policy (cmc_grants.hpp) without a device.
void check_grants() {
    auto total = [](const std::vector<GrantShare>& g) {
        uint64_t t = 0;
        for (const GrantShare& x : g) t += x.trials;
        return t;
    };
    auto of = [](const std::vector<GrantShare>& g, uint32_t id) {
        for (const GrantShare& x : g)
            if (x.id == id) return x.trials;
        return uint64_t(0);
    };
    // three jobs of 4096 trials (batches of 1024) at 100 blocks per trial;
    // job 7 arrived first, job 3 last
    std::vector<GrantCandidate> jobs = {{3, 0, 4096, 10, 100.0, 0.0, 30},
                                        {5, 0, 4096, 10, 100.0, 0.0, 20},
                                        {7, 0, 4096, 10, 100.0, 0.0, 10}};
    // all in arrival order: the step grows to an eighth of the backlog
    // (153,600 blocks); the oldest takes what one grant holds (a batch), the
    // next the rest
    auto g = grant_shares(jobs, 150000, 1.0, 1u << 20);
    require(of(g, 7) == 1024 && of(g, 5) == 512 && of(g, 3) == 0, "arrival order fills the oldest first");
    // a grant never crosses a batch boundary, even when more work is asked for
    jobs[2].next = 1000;
    g = grant_shares(jobs, 1u << 30, 1.0, 1u << 20);
    require(of(g, 7) == 24, "a grant stops at the end of its batch");
    jobs[2].next = 0;
    // shortest remaining work first when nothing goes in arrival order: job 3
    // (96 trials left) is served whole, the step (an eighth of the 828,800-
    // block backlog) gives the rest, 940 trials, to the next shortest
    jobs[0].next = 4000;
    g = grant_shares(jobs, 20000, 0.0, 1u << 20);
    require(of(g, 3) == 96 && of(g, 7) + of(g, 5) == 940, "shortest remaining work goes first");
    // the trial cap holds
    g = grant_shares(jobs, 1u << 30, 0.5, 300);
    require(total(g) == 300, "no more than max_trials in one step");
    // a step covers 2.5x the slowest trial's latency even if less was asked
    std::vector<GrantCandidate> slow = {{1, 0, 1u << 16, 16, 10.0, 4000.0, 1}};
    g = grant_shares(slow, 10, 1.0, 1u << 20);
    require(of(g, 1) == 1000, "the step is at least 2.5x one trial's latency");
    // heaviest trials first in the table
    std::vector<GrantCandidate> mix = {{1, 0, 64, 6, 10.0, 0.0, 1}, {2, 0, 64, 6, 1000.0, 0.0, 2},
                                       {3, 0, 64, 6, 100.0, 0.0, 3}};
    g = grant_shares(mix, 1u << 30, 0.95, 1u << 20);
    require(g.size() == 3 && g[0].id == 2 && g[1].id == 3 && g[2].id == 1, "heaviest trials first");
    // a finished job gets nothing
    mix[1].next = mix[1].budget;
    g = grant_shares(mix, 1u << 30, 0.95, 1u << 20);
    require(of(g, 2) == 0 && g.size() == 2, "no trials past a budget");
}

int main(int argc, char** argv) {
    try {
        const fs::path base = fs::absolute(argc > 1 ? argv[1] : "host_test_data");
        const fs::path root = base / ("run_" + std::to_string(steady_ns()));
        fs::create_directories(root);
        check_keys();
        check_grants();
        check_pause(root);
        check_journals(root);
        check_k_extension(root);
        check_locks_and_parameters(root);
        fs::remove_all(root);
        std::cout << "ALL HOST TESTS PASSED (" << g_checks << " checks)\n";
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "TEST FAILURE: " << e.what() << '\n';
        return 1;
    }
}
