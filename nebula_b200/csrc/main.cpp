// nebula_b200: command-line drop-in for Nebula's nebula_gpu.
//
//   nebula_b200 [options] <geometry.tri> <primaries.pri> mat0.mat ... matN.mat > detected.bin
//
// Same options, inputs and output as source/gpu_main.cu:221-440: detected
// electrons are written to stdout as 36-byte records {pos, dir, E, px, py};
// progress and timing go to stderr; usage errors exit with status 1.  The
// host side calls the library only through the C ABI of include/nbx.h.
// --prescan-size and --batch-factor are accepted for compatibility: the
// persistent queue needs no prescan (gpu_main.cu:109-175 sized frames with
// it); they only size the batches of the --energy-deposit mode.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iostream>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "nbx.h"

namespace {

// --key=value / --key value parser with the reference's rules
// (source/common/cli_params.h:54-90): unknown keys are errors.
struct Cli {
    std::map<std::string, std::pair<std::string, std::string>> opts;   // key -> (description, value)
    std::vector<std::string> positional;
    std::string program;
    void add(const std::string& k, const std::string& d, const std::string& v) { opts[k] = {d, v}; }
    void parse(int argc, char** argv) {
        program = argv[0];
        for (int i = 1; i < argc; ++i) {
            std::string item = argv[i];
            if (item.size() >= 2 && item[0] == '-' && item[1] == '-') {
                std::string key, value;
                const auto split = item.find('=', 2);
                if (split == std::string::npos) {
                    key = item.substr(2);
                    value = (++i < argc) ? argv[i] : "";
                    if (value == "=") value = (++i < argc) ? argv[i] : "";
                } else {
                    key = item.substr(2, split - 2);
                    value = item.substr(split + 1);
                }
                auto it = opts.find(key);
                if (it == opts.end()) throw std::runtime_error("Unexpected key '" + key + "'");
                it->second.second = value;
            } else {
                positional.push_back(item);
            }
        }
    }
    void usage(std::ostream& out) const {
        out << "Usage: " << program << " [options] <geometry.tri> <primaries.pri> [material0.mat] .. [materialN.mat]\n"
            << "Options:\n";
        for (auto& o : opts) out << "\t--" << o.first << ": " << o.second.first << " [" << o.second.second << "]\n";
    }
    template <typename T>
    T get(const std::string& k) const {
        std::istringstream ss(opts.at(k).second);
        T v{};
        ss >> v;
        return v;
    }
};

template <>
bool Cli::get<bool>(const std::string& k) const {
    const std::string& v = opts.at(k).second;
    return v == "1" || v == "true" || v == "True" || v == "yes";
}

struct Timer {
    std::vector<std::pair<std::string, double>> rows;
    std::chrono::steady_clock::time_point t0;
    void start() { t0 = std::chrono::steady_clock::now(); }
    void stop(const std::string& name) {
        rows.emplace_back(name, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    void print() const {
        size_t w = 0;
        for (auto& r : rows) w = std::max(w, r.first.size());
        std::fprintf(stderr, "Timing (seconds):\n");
        for (auto& r : rows) std::fprintf(stderr, "%*s: %.3f\n", int(w), r.first.c_str(), r.second);
    }
};

uint64_t morton(uint16_t x, uint16_t y, uint16_t z) {
    uint64_t m = 0;
    for (unsigned i = 0; i < 16; ++i) {
        m |= (uint64_t(x) & (uint64_t(1) << i)) << (2 * i + 0);
        m |= (uint64_t(y) & (uint64_t(1) << i)) << (2 * i + 1);
        m |= (uint64_t(z) & (uint64_t(1) << i)) << (2 * i + 2);
    }
    return m;
}

int die(nbx_ctx* ctx, int rc, const char* what) {
    std::fprintf(stderr, "Error: %s: %s (%s)\n", what, nbx_error_string(rc), ctx ? nbx_last_error(ctx) : "");
    return 1;
}

// Counts of the reference loader's warnings (io/load_pri_file.cpp:120-176).
struct PriWarnings {
    const nbx_octree* oct;
    float max_energy;
    uint64_t outside = 0, low = 0, high = 0, dir0 = 0;
    void add(const nbx_record* pri, uint64_t n) {
        const float eps = 10 * 1.1920928955078125e-07f;
        for (uint64_t i = 0; i < n; ++i) {
            const nbx_record& r = pri[i];
            bool inside = true;
            for (int k = 0; k < 3; ++k)
                inside = inside && r.pos[k] > oct->center[k] - oct->halfsize[k] &&
                         r.pos[k] < oct->center[k] + oct->halfsize[k];
            outside += !inside;
            low += !(r.E > eps);
            high += r.E > max_energy;
            dir0 += !(std::fabs(r.dir[0]) > eps || std::fabs(r.dir[1]) > eps || std::fabs(r.dir[2]) > eps);
        }
    }
    void print() const {
        if (outside) std::fprintf(stderr, "WARNING: %llu primary electrons starting outside geometry.\n", (unsigned long long)outside);
        if (low) std::fprintf(stderr, "WARNING: %llu primary electrons starting with low kinetic energy.\n", (unsigned long long)low);
        if (high)
            std::fprintf(stderr, "WARNING: %llu primary electrons starting with kinetic energy higher than what is "
                                 "available in the material files. Limit is %g keV.\n", (unsigned long long)high, max_energy / 1000);
        if (dir0) std::fprintf(stderr, "WARNING: %llu primary electrons start with unphysical direction vector.\n", (unsigned long long)dir0);
    }
};

// Primaries either read whole (for sorting) or streamed from the file in
// batches; read(first, n, out) copies records first .. first + n - 1 with a
// positional read, so batches can be read by several threads at once.
struct PriSource {
    nbx_record* all = nullptr;
    uint64_t count = 0;
    int fd = -1;
    bool open(const std::string& path, bool whole) {
        if (whole) return nbx_load_pri(path.c_str(), &all, &count) == NBX_OK && count > 0;
        fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) return false;
        struct stat st;
        if (fstat(fd, &st) != 0) return false;
        const long long size = st.st_size;
        if (size <= 0 || size % 36 != 0) return false;   // "Unexpected end of primaries file"
        count = uint64_t(size) / 36;
        return true;
    }
    bool read(uint64_t first, uint64_t n, nbx_record* out) const {
        if (all) {
            std::memcpy(out, all + first, sizeof(nbx_record) * n);
            return true;
        }
        char* dst = reinterpret_cast<char*>(out);
        uint64_t left = 36 * n, off = 36 * first;
        while (left) {
            const ssize_t got = ::pread(fd, dst, size_t(std::min<uint64_t>(left, 1ull << 30)), off_t(off));
            if (got <= 0) return false;
            dst += got;
            off += uint64_t(got);
            left -= uint64_t(got);
        }
        return true;
    }
    ~PriSource() {
        if (all) nbx_free(all);
        if (fd >= 0) ::close(fd);
    }
};

// Hand-off of buffers between threads: pop() waits for an item; once the
// queue is closed it returns what is left, then nullptr.
template <typename T>
class Handoff {
public:
    void push(T* x) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(x);
        }
        cv_.notify_one();
    }
    T* pop() {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !q_.empty() || closed_; });
        if (q_.empty()) return nullptr;
        T* x = q_.front();
        q_.pop_front();
        return x;
    }
    void close() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            closed_ = true;
        }
        cv_.notify_all();
    }

private:
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<T*> q_;
    bool closed_ = false;
};

// One batch of primaries on the host: the particles and batch-relative tags
// in page-locked memory (so nbx_stage's copy overlaps a running batch) and
// each primary's pixel, which its detected records carry.
struct HostBatch {
    uint64_t first = 0, n = 0;
    nbx_particle* part = nullptr;
    uint32_t* tags = nullptr;
    std::vector<int32_t> px, py;
};

// Detected records of one batch on their way to the output: read back from
// the device into page-locked memory (the library's layout; the rare records
// beyond `cap` into `more`) and turned into the reference's 36-byte records
// by the writer thread, with the pixel of the primary each one came from.
struct OutBatch {
    nbx_detected* det = nullptr;
    uint64_t cap = 0, n = 0;
    std::vector<nbx_detected> more;
    HostBatch* src = nullptr;
};

}  // namespace

int main(int argc, char** argv) {
    std::fprintf(stderr, "This is nebula_b200 (Nebula-compatible, version %d.%d.%d)\n\n", NBX_VERSION_MAJOR,
                 NBX_VERSION_MINOR, NBX_VERSION_PATCH);
    Cli p;
    p.add("energy-threshold", "Lowest energy to simulate", "0");
    p.add("capacity", "Electron capacity on the GPU (primaries per device run)", "4000000");
    p.add("prescan-size", "Number of electrons to use for prescan", "1000");
    p.add("batch-factor", "Multiplication factor for electron batch size", "0.9");
    p.add("seed", "Random seed", std::to_string(0x78c7e39b));
    p.add("sort-primaries", "Sort primary electrons before simulation", "0");
    p.add("device", "CUDA device ordinal", "0");
    p.add("streams", "Device contexts, each with its own pipeline of batches (one with --energy-deposit)", "1");
    p.add("inelastic", "Inelastic model: kieft (Kieft & Bosch) or penn (full Penn, the reference's stock build)",
          "kieft");
    p.add("energy-deposit", "Also write energy deposits, as the reference's nebula_cpu_energydep", "0");
    p.add("detect-filename", "With --energy-deposit: file for detected electrons", "detected.bin");
    p.add("deposit-filename", "With --energy-deposit: file for energy deposits", "stdout");
    try {
        p.parse(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        p.usage(std::cerr);
        return 1;
    }
    const float energy_threshold = p.get<float>("energy-threshold");
    const uint64_t capacity = p.get<uint64_t>("capacity");
    const uint32_t prescan = p.get<uint32_t>("prescan-size");
    const float batch_factor = p.get<float>("batch-factor");
    const uint32_t seed = p.get<uint32_t>("seed");
    const bool sort_primaries = p.get<bool>("sort-primaries");
    const int device = p.get<int>("device");
    const int streams = p.get<int>("streams");
    const std::string inelastic = p.get<std::string>("inelastic");
    const bool energy_deposit = p.get<bool>("energy-deposit");
    const std::string detect_filename = p.get<std::string>("detect-filename");
    const std::string deposit_filename = p.get<std::string>("deposit-filename");
    if (p.positional.size() < 3 || capacity == 0 || prescan == 0 || batch_factor <= 0 || streams < 1 || streams > 8 ||
        (inelastic != "kieft" && inelastic != "penn")) {
        p.usage(std::cerr);
        return 1;
    }
    Timer timer;

    // Geometry (gpu_main.cu:287-325)
    std::fprintf(stderr, "Loading geometry...\n");
    timer.start();
    nbx_triangle* tris = nullptr;
    uint64_t n_tris = 0;
    int rc = nbx_load_tri(p.positional[0].c_str(), &tris, &n_tris);
    timer.stop("Loading triangles");
    if (rc != NBX_OK || n_tris == 0) {
        std::fprintf(stderr, "Error: could not load triangles!\n");
        p.usage(std::cerr);
        return 1;
    }
    {
        int max_material = -1;
        for (uint64_t i = 0; i < n_tris; ++i) max_material = std::max({max_material, tris[i].mat_in, tris[i].mat_out});
        const int provided = int(p.positional.size()) - 2;
        if (max_material > provided - 1) {
            std::fprintf(stderr, "Error: not enough materials provided for this geometry!\n  Expected %d materials, %d provided.\n",
                         max_material + 1, provided);
            return 1;
        }
        if (max_material < provided - 1)
            std::fprintf(stderr, "Warning: too many materials provided for this geometry!\n  Expected %d materials, %d provided.\n",
                         max_material + 1, provided);
    }
    timer.start();
    nbx_octree* oct = nullptr;
    rc = nbx_octree_build(tris, n_tris, &oct);
    nbx_free(tris);
    if (rc != NBX_OK) return die(nullptr, rc, "octree build");
    timer.stop("Building acceleration structure");

    // Materials (gpu_main.cu:332-349)
    std::fprintf(stderr, "Loading materials...\n");
    timer.start();
    std::vector<nbx_material*> mats;
    float max_energy = INFINITY;
    for (size_t i = 2; i < p.positional.size(); ++i) {
        nbx_material* m = nullptr;
        rc = nbx_material_load(p.positional[i].c_str(), &m);
        if (rc != NBX_OK) {
            std::fprintf(stderr, "Error: could not load material %s\n", p.positional[i].c_str());
            return 1;
        }
        std::fprintf(stderr, "  Material %zu:\n    Name: %s\n", i - 2, m->name);
        max_energy = std::min(max_energy, inelastic == "penn" ? m->penn_max_energy : m->max_energy);
        mats.push_back(m);
    }
    timer.stop("Loading materials");

    // Primaries (gpu_main.cu:352-380, io/load_pri_file.cpp:72-229).  Without
    // --sort-primaries the file is streamed batch by batch (a 7.5 GB scan
    // never sits in host memory); the reference's warnings are counted as the
    // batches go by and printed once the last batch is read.  Sorting needs
    // every primary, so --sort-primaries loads the whole file first.
    std::fprintf(stderr, "Loading primary electrons...\n");
    timer.start();
    PriWarnings warn{oct, max_energy};
    PriSource src;
    if (!src.open(p.positional[1], sort_primaries)) {
        std::fprintf(stderr, "Error: could not load primary electrons!\n");
        p.usage(std::cerr);
        return 1;
    }
    const uint64_t n_pri = src.count;
    if (sort_primaries) {
        nbx_record* pri = src.all;
        warn.add(pri, n_pri);
        warn.print();
        // Morton order of the start positions (io/load_pri_file.cpp:186-229)
        float vmin[3], vmax[3];
        for (int k = 0; k < 3; ++k) vmin[k] = vmax[k] = pri[0].pos[k];
        for (uint64_t i = 0; i < n_pri; ++i)
            for (int k = 0; k < 3; ++k) {
                vmin[k] = std::min(vmin[k], pri[i].pos[k]);
                vmax[k] = std::max(vmax[k], pri[i].pos[k]);
            }
        std::vector<uint64_t> key(n_pri);
        for (uint64_t i = 0; i < n_pri; ++i) {
            uint16_t q[3];
            for (int k = 0; k < 3; ++k) {
                const float sz = vmax[k] - vmin[k];
                q[k] = uint16_t((pri[i].pos[k] - vmin[k]) / sz * 65535);
            }
            key[i] = morton(q[0], q[1], q[2]);
        }
        std::vector<uint64_t> perm(n_pri);
        std::iota(perm.begin(), perm.end(), 0);
        std::stable_sort(perm.begin(), perm.end(), [&](uint64_t a, uint64_t b) { return key[a] < key[b]; });
        std::vector<nbx_record> sorted(n_pri);
        for (uint64_t i = 0; i < n_pri; ++i) sorted[i] = pri[perm[i]];
        std::memcpy(pri, sorted.data(), sizeof(nbx_record) * n_pri);
    }
    timer.stop("Loading primary electrons");

    // Device context
    nbx_config cfg;
    nbx_config_default(&cfg);
    cfg.device = device;
    cfg.seed = seed;
    cfg.energy_threshold = energy_threshold;
    cfg.inelastic_model = inelastic == "penn" ? NBX_INELASTIC_FULL_PENN : NBX_INELASTIC_KIEFT;
    cfg.record_detected = 1;
    cfg.record_capacity = 1ull << 24;
    cfg.record_deposits = energy_deposit ? 1 : 0;
    // --streams contexts on the one device, each running its own pipeline
    // of batches (below); one keeps the device busy already.
    const int n_ctx = energy_deposit ? 1 : streams;
    std::vector<nbx_ctx*> ctxs;
    for (int k = 0; k < n_ctx; ++k) {
        nbx_ctx* c = nullptr;
        rc = nbx_create(&c, &cfg);
        if (rc != NBX_OK) return die(nullptr, rc, "nbx_create");
        ctxs.push_back(c);
        if ((rc = nbx_set_geometry(c, oct)) != NBX_OK) return die(c, rc, "set_geometry");
        for (auto* m : mats)
            if ((rc = nbx_add_material(c, m)) != NBX_OK) return die(c, rc, "add_material");
    }
    std::fprintf(stderr, "\nLoaded %llu triangles.\nLoaded %llu primaries.\nLoaded %zu materials.\n\n",
                 (unsigned long long)oct->n_triangles, (unsigned long long)n_pri, mats.size());

    // Simulation: batches of `capacity` primaries, detected records streamed out.
    // With --energy-deposit (cpu_energydep.cpp:156-214): detected electrons go
    // to --detect-filename and 28-byte deposit records {x, y, z, E, dE, px, py}
    // to --deposit-filename; the first batch (--prescan-size primaries) measures
    // deposits per primary, and later batches are sized to fit the device's
    // deposit buffer (times --batch-factor).
    FILE* detect_out = stdout;
    FILE* deposit_out = nullptr;
    if (energy_deposit) {
        detect_out = detect_filename == "stdout" ? stdout : std::fopen(detect_filename.c_str(), "wb");
        deposit_out = deposit_filename == "stdout" ? stdout : std::fopen(deposit_filename.c_str(), "wb");
        if (!detect_out || !deposit_out) {
            std::fprintf(stderr, "Error: could not open the output files\n");
            return 1;
        }
    }
    struct DepositRecord {
        float x, y, z, E, dE;
        int32_t px, py;
    };
    static_assert(sizeof(DepositRecord) == 28, "deposit record layout");
    const uint64_t dep_capacity = uint64_t(1) << 27;   // nbx_config default

    // Energy-deposit mode: one context runs the batches in turn on this
    // thread.  It reads each batch with a positional read, runs it, writes
    // its records, then sizes the next batch from the deposits per primary
    // seen so far.  In every mode a batch's primaries keep their global index
    // as the uid of their random streams, so the records depend neither on
    // the batch size nor on the number of contexts; only their order in the
    // output does, as with the reference's worker threads.  Tags are
    // batch-relative.
    struct Batch {
        uint64_t first = 0, n = 0;
        std::vector<nbx_record> pri;
        std::vector<nbx_particle> part;
        std::vector<uint32_t> tags;
    };
    std::mutex fail_mu;
    uint64_t done = 0;
    uint64_t batch = std::max<uint64_t>(capacity, 1);
    if (energy_deposit) batch = std::min<uint64_t>(batch, std::max<uint32_t>(prescan, 1));
    int failed_rc = NBX_OK;
    std::string failed_what;
    nbx_ctx* failed_ctx = nullptr;
    auto fail_with = [&](nbx_ctx* c, int code, const char* what) {
        std::lock_guard<std::mutex> lk(fail_mu);
        if (failed_rc == NBX_OK) {
            failed_rc = code;
            failed_what = what;
            failed_ctx = c;
        }
    };
    auto deposit_loop = [&](nbx_ctx* c) {
        Batch b;
        std::vector<nbx_detected> det(1u << 20);
        std::vector<nbx_deposit> dep(1u << 20);
        std::vector<nbx_record> out;
        std::vector<DepositRecord> dep_out;
        for (uint64_t first = 0; first < n_pri; first += b.n) {
            b.first = first;
            b.n = std::min(batch, n_pri - first);
            b.pri.resize(b.n);
            if (!src.read(b.first, b.n, b.pri.data())) {
                std::fprintf(stderr, "Error: could not read primary electrons!\n");
                return fail_with(c, NBX_ERR_FORMAT, "primaries");
            }
            if (!sort_primaries) warn.add(b.pri.data(), b.n);
            b.part.resize(b.n);
            b.tags.resize(b.n);
            for (uint64_t i = 0; i < b.n; ++i) {
                std::memcpy(b.part[i].pos, b.pri[i].pos, 12);
                std::memcpy(b.part[i].dir, b.pri[i].dir, 12);
                b.part[i].E = b.pri[i].E;
                b.tags[i] = uint32_t(i);
            }
            int r;
            uint64_t acc = 0;
            if ((r = nbx_set_uid_base(c, b.first)) != NBX_OK) return fail_with(c, r, "uid base");
            if ((r = nbx_push(c, b.part.data(), b.tags.data(), b.n, &acc)) != NBX_OK) return fail_with(c, r, "push");
            if ((r = nbx_run(c)) != NBX_OK) return fail_with(c, r, "run");
            out.clear();
            for (;;) {
                uint64_t got = 0;
                if ((r = nbx_flush_detected(c, det.data(), det.size(), &got)) != NBX_OK) return fail_with(c, r, "flush");
                if (got == 0) break;
                const size_t base = out.size();
                out.resize(base + got);
                for (uint64_t i = 0; i < got; ++i) {
                    nbx_record& o = out[base + i];
                    std::memcpy(o.pos, det[i].pos, 12);
                    std::memcpy(o.dir, det[i].dir, 12);
                    o.E = det[i].E;
                    o.px = b.pri[det[i].tag].px;
                    o.py = b.pri[det[i].tag].py;
                }
            }
            dep_out.clear();
            for (;;) {
                uint64_t got = 0;
                if ((r = nbx_flush_deposits(c, dep.data(), dep.size(), &got)) != NBX_OK)
                    return fail_with(c, r, "flush deposits");
                if (got == 0) break;
                const size_t base = dep_out.size();
                dep_out.resize(base + got);
                for (uint64_t i = 0; i < got; ++i) {
                    const nbx_deposit& d = dep[i];
                    const nbx_record& rec = b.pri[d.tag];
                    dep_out[base + i] = {d.pos[0], d.pos[1], d.pos[2], d.E, d.dE, rec.px, rec.py};
                }
            }
            nbx_stats st;
            nbx_get_stats(c, &st);
            if (st.deposits_dropped) {
                std::fprintf(stderr, "\nError: %llu energy deposits did not fit the device buffer; lower --batch-factor\n",
                             (unsigned long long)st.deposits_dropped);
                return fail_with(c, NBX_ERR_CAPACITY, "deposit buffer");
            }
            // size the next batches from the deposits per primary seen so far
            const double per_primary = double(dep_out.size()) / double(b.n);
            const double fit = batch_factor * double(dep_capacity) / std::max(per_primary, 1.0);
            batch = std::max<uint64_t>(1, std::min<uint64_t>(std::max<uint64_t>(capacity, 1), uint64_t(fit)));
            if (!out.empty()) std::fwrite(out.data(), sizeof(nbx_record), out.size(), detect_out);
            if (!dep_out.empty()) std::fwrite(dep_out.data(), sizeof(DepositRecord), dep_out.size(), deposit_out);
            done += b.n;
            std::fprintf(stderr, " \rProgress %.2f%%", 100.0 * double(done) / double(n_pri));
        }
    };

    // Plain mode: a pipeline that keeps the device busy.  A reader thread
    // reads batches ahead of the device into page-locked buffers.  Each
    // context's thread starts the copy of its next batch (nbx_stage) before it
    // runs the current one, so the copy overlaps the run (the reference's
    // frame loop overlaps its copies the same way, gpu_driver.inl:167-306);
    // after the run it collects the batch's records and queues the next batch
    // (nbx_push_staged).  A writer thread writes the records in the order the
    // batches finish.  The device only waits for the record read-back and the
    // queueing between two runs.
    Handoff<HostBatch> ready, free_batches;
    Handoff<OutBatch> written, free_out;
    std::vector<HostBatch> host_batches(energy_deposit ? 0 : size_t(2 * n_ctx + 3));
    std::vector<OutBatch> out_batches(energy_deposit ? 0 : size_t(2 * n_ctx + 2));
    auto close_all = [&] {
        ready.close();
        free_batches.close();
        written.close();
        free_out.close();
    };
    // Page-locked buffers are allocated where they are first needed, off the
    // device's critical path: the reader's on first use, the read-back
    // buffers by the writer thread as it starts.
    const uint64_t buf_n = std::min(batch, n_pri);
    auto reader = [&] {
        std::vector<nbx_record> raw;
        for (uint64_t first = 0; first < n_pri; first += batch) {
            HostBatch* b = free_batches.pop();
            if (!b) return;
            if (!b->part) {
                void* p = nullptr;
                void* t = nullptr;
                if (nbx_host_alloc(sizeof(nbx_particle) * buf_n, &p) != NBX_OK ||
                    nbx_host_alloc(sizeof(uint32_t) * buf_n, &t) != NBX_OK) {
                    nbx_host_free(p);
                    fail_with(nullptr, NBX_ERR_OOM, "page-locked batch buffers (lower --capacity)");
                    return close_all();
                }
                b->part = static_cast<nbx_particle*>(p);
                b->tags = static_cast<uint32_t*>(t);
            }
            b->first = first;
            b->n = std::min(batch, n_pri - first);
            raw.resize(b->n);
            if (!src.read(first, b->n, raw.data())) {
                std::fprintf(stderr, "Error: could not read primary electrons!\n");
                fail_with(nullptr, NBX_ERR_FORMAT, "primaries");
                return close_all();
            }
            if (!sort_primaries) warn.add(raw.data(), b->n);
            b->px.resize(b->n);
            b->py.resize(b->n);
            for (uint64_t i = 0; i < b->n; ++i) {
                std::memcpy(b->part[i].pos, raw[i].pos, 12);
                std::memcpy(b->part[i].dir, raw[i].dir, 12);
                b->part[i].E = raw[i].E;
                b->tags[i] = uint32_t(i);
                b->px[i] = raw[i].px;
                b->py[i] = raw[i].py;
            }
            ready.push(b);
        }
        for (int k = 0; k < n_ctx; ++k) ready.push(nullptr);   // one end mark per context
    };
    auto pipeline = [&](nbx_ctx* c) {
        auto failed = [&](int code, const char* what) {
            fail_with(c, code, what);
            close_all();
        };
        HostBatch* cur = ready.pop();
        if (!cur) return;
        int r;
        if ((r = nbx_set_uid_base(c, cur->first)) != NBX_OK) return failed(r, "uid base");
        if ((r = nbx_stage(c, cur->part, cur->tags, cur->n)) != NBX_OK) return failed(r, "stage");
        if ((r = nbx_push_staged(c, nullptr)) != NBX_OK) return failed(r, "push");
        for (;;) {
            HostBatch* next = ready.pop();
            if (next && (r = nbx_stage(c, next->part, next->tags, next->n)) != NBX_OK) return failed(r, "stage");
            if ((r = nbx_run(c)) != NBX_OK) return failed(r, "run");
            OutBatch* o = free_out.pop();
            if (!o) return;
            o->n = 0;
            o->more.clear();
            o->src = cur;
            for (;;) {
                uint64_t got = 0;
                if (o->n < o->cap) {
                    if ((r = nbx_flush_detected(c, o->det + o->n, o->cap - o->n, &got)) != NBX_OK)
                        return failed(r, "flush");
                    o->n += got;
                } else {
                    const size_t base = o->more.size();
                    o->more.resize(base + (1u << 20));
                    if ((r = nbx_flush_detected(c, o->more.data() + base, 1u << 20, &got)) != NBX_OK)
                        return failed(r, "flush");
                    o->more.resize(base + got);
                }
                if (got == 0) break;
            }
            written.push(o);
            if (!next) return;
            if ((r = nbx_set_uid_base(c, next->first)) != NBX_OK) return failed(r, "uid base");
            if ((r = nbx_push_staged(c, nullptr)) != NBX_OK) return failed(r, "push");
            cur = next;
        }
    };
    auto writer = [&] {
        for (OutBatch& o : out_batches) {
            void* d = nullptr;
            if (nbx_host_alloc(sizeof(nbx_detected) * buf_n, &d) != NBX_OK) {
                fail_with(nullptr, NBX_ERR_OOM, "page-locked record buffers (lower --capacity)");
                return close_all();
            }
            o.det = static_cast<nbx_detected*>(d);
            o.cap = buf_n;
            free_out.push(&o);
        }
        std::vector<nbx_record> out;
        for (;;) {
            OutBatch* o = written.pop();
            if (!o) return;
            const HostBatch* b = o->src;
            out.resize(o->n + o->more.size());
            for (size_t i = 0; i < out.size(); ++i) {
                const nbx_detected& d = i < o->n ? o->det[i] : o->more[i - o->n];
                nbx_record& rec = out[i];
                std::memcpy(rec.pos, d.pos, 12);
                std::memcpy(rec.dir, d.dir, 12);
                rec.E = d.E;
                rec.px = b->px[d.tag];
                rec.py = b->py[d.tag];
            }
            if (!out.empty()) std::fwrite(out.data(), sizeof(nbx_record), out.size(), detect_out);
            done += b->n;
            std::fprintf(stderr, " \rProgress %.2f%%", 100.0 * double(done) / double(n_pri));
            free_batches.push(o->src);
            free_out.push(o);
        }
    };

    timer.start();
    if (energy_deposit) {
        deposit_loop(ctxs[0]);
    } else {
        for (HostBatch& b : host_batches) free_batches.push(&b);
        std::thread out_thread(writer);
        std::vector<std::thread> threads;
        threads.emplace_back(reader);
        for (nbx_ctx* c : ctxs) threads.emplace_back(pipeline, c);
        for (auto& t : threads) t.join();
        written.close();   // every context has handed over its last batch
        out_thread.join();
    }
    if (failed_rc != NBX_OK) {
        const int r = die(failed_ctx, failed_rc, failed_what.c_str());
        for (nbx_ctx* c : ctxs) nbx_destroy(c);
        return r;
    }
    std::fflush(stdout);
    if (!sort_primaries) {
        std::fprintf(stderr, "\n");
        warn.print();
    }
    if (energy_deposit) {
        if (detect_out != stdout) std::fclose(detect_out);
        if (deposit_out != stdout) std::fclose(deposit_out);
    }
    timer.stop("Simulation");
    nbx_stats st{};
    for (nbx_ctx* c : ctxs) {
        nbx_stats one;
        nbx_get_stats(c, &one);
        st.events_elastic += one.events_elastic;
        st.events_inelastic += one.events_inelastic;
        st.events_boundary += one.events_boundary;
        st.detected += one.detected;
        st.records_dropped += one.records_dropped;
    }
    std::fprintf(stderr, "\n\nSimulation successful!\n  events: %llu elastic, %llu inelastic, %llu boundary; %llu detected",
                 (unsigned long long)st.events_elastic, (unsigned long long)st.events_inelastic,
                 (unsigned long long)st.events_boundary, (unsigned long long)st.detected);
    if (st.records_dropped) std::fprintf(stderr, " (%llu records dropped)", (unsigned long long)st.records_dropped);
    std::fprintf(stderr, "\n\n");
    timer.print();
    for (nbx_ctx* c : ctxs) nbx_destroy(c);
    for (HostBatch& b : host_batches) {
        nbx_host_free(b.part);
        nbx_host_free(b.tags);
    }
    for (OutBatch& o : out_batches) nbx_host_free(o.det);
    for (auto* m : mats) nbx_material_free(m);
    nbx_octree_free(oct);
    return 0;
}
