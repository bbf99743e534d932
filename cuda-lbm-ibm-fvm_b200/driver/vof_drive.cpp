// vof_drive.cpp -- drop-in for voftrial1.cu's main() (voftrial1.cu:1228-1422)
// on the vof C-ABI: the same command line (-ic, --nstep, --max_steps), the same
// initial condition, console lines, dump files and timing line, with the time
// loop stepping through vof_run (captured CUDA graphs) and the dumps taken off
// the critical path.
//
// Dumps.  The reference stops the GPU at every dump step (cudaDeviceSynchronize
// + a blocking cudaMemcpy) and formats 8.2 M values through iostreams before
// the next step starts (voftrial1.cu:1403-1411, 907-941).  Here a dump is a
// device-to-device copy of F into a staging buffer (reference layout) on the
// solver's stream; a side stream copies the staging buffer to pinned host
// memory once it is ready, and a writer thread formats and writes the file
// while the solver keeps stepping.  Two staging/pinned pairs rotate; the
// solver waits only when both are still being written.  ASCII output is
// byte-identical to write_legacy_vtk (same header, values as printf("%.8g")),
// formatted by a pool of threads; --vtk binary writes the same header with
// BINARY and big-endian float32 data (the legacy VTK binary convention).
//
// Additions to the reference's options (it hardcodes them): grid size,
// gravity, dt, Jacobi sweeps, solver mode, output directory and format, an
// initial F read from a raw float32 file in the reference layout, and a final
// dump of every state field as raw float32.
#include <cuda_runtime.h>

#include <algorithm>
#include <charconv>
#include <chrono>
#include <condition_variable>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <iomanip>
#include <iostream>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "vof.h"

namespace {

volatile std::sig_atomic_t g_stop = 0;
void handle_signal(int) { g_stop = 1; }

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

size_t idx3d(int i, int j, int k, int nxTot, int nyTot) {
    return ((size_t)k * (size_t)nyTot + (size_t)j) * (size_t)nxTot + (size_t)i;
}

// set_init_F_kernel (voftrial1.cu:72-93) on the host: the same float
// expressions, evaluated at every cell including the ghosts.  ic 2 and 3 are
// accepted and leave F = 0, as in the reference.
void init_F(const vof_params& p, int ic, std::vector<float>& F) {
    const int nxTot = p.nx + 2, nyTot = p.ny + 2, nzTot = p.nz + 2;
    F.assign((size_t)nxTot * nyTot * nzTot, 0.0f);
    if (ic != 1) return;
    for (int k = 0; k < nzTot; ++k)
        for (int j = 0; j < nyTot; ++j)
            for (int i = 0; i < nxTot; ++i) {
                const float x = static_cast<float>(clampi(i - 1, 0, p.nx)) * p.dx;
                const float y = static_cast<float>(clampi(j - 1, 0, p.ny)) * p.dy;
                const float z = static_cast<float>(clampi(k - 1, 0, p.nz)) * p.dz;
                if ((x >= 0.0f && x <= p.Lx / 3.0f) && (y >= 0.0f && y <= p.Ly / 2.0f) &&
                    (z >= 0.0f && z <= p.Lz / 3.0f))
                    F[idx3d(i, j, k, nxTot, nyTot)] = 1.0f;
            }
}

// apply_bc_F (voftrial1.cu:1122-1135, kernels 1053-1105): zero-gradient
// ghosts, j then i then k, each over the full extent of the other two axes.
void bc_F(const vof_params& p, std::vector<float>& F) {
    const int nxTot = p.nx + 2, nyTot = p.ny + 2, nzTot = p.nz + 2;
    for (int k = 0; k < nzTot; ++k)
        for (int i = 0; i < nxTot; ++i) {
            F[idx3d(i, 0, k, nxTot, nyTot)] = F[idx3d(i, 1, k, nxTot, nyTot)];
            F[idx3d(i, p.ny + 1, k, nxTot, nyTot)] = F[idx3d(i, p.ny, k, nxTot, nyTot)];
        }
    for (int k = 0; k < nzTot; ++k)
        for (int j = 0; j < nyTot; ++j) {
            F[idx3d(0, j, k, nxTot, nyTot)] = F[idx3d(1, j, k, nxTot, nyTot)];
            F[idx3d(p.nx + 1, j, k, nxTot, nyTot)] = F[idx3d(p.nx, j, k, nxTot, nyTot)];
        }
    for (int j = 0; j < nyTot; ++j)
        for (int i = 0; i < nxTot; ++i) {
            F[idx3d(i, j, 0, nxTot, nyTot)] = F[idx3d(i, j, 1, nxTot, nyTot)];
            F[idx3d(i, j, p.nz + 1, nxTot, nyTot)] = F[idx3d(i, j, p.nz, nxTot, nyTot)];
        }
}

enum class Vtk { Ascii, Binary, None };

// The header of write_legacy_vtk (voftrial1.cu:918-932): SPACING printed with
// the stream's default precision (6 significant digits), before the data's
// setprecision(8).
std::string vtk_header(int nxTot, int nyTot, int nzTot, bool binary) {
    const float sx = 1.0f / static_cast<float>(nxTot - 1);
    const float sy = 1.0f / static_cast<float>(nyTot - 1);
    const float sz = 1.0f / static_cast<float>(nzTot - 1);
    std::ostringstream out;
    out << "# vtk DataFile Version 3.0\n";
    out << "3D VOF field\n";
    out << (binary ? "BINARY\n" : "ASCII\n");
    out << "DATASET STRUCTURED_POINTS\n";
    out << "DIMENSIONS " << nxTot << " " << nyTot << " " << nzTot << "\n";
    out << "ORIGIN 0 0 0\n";
    out << "SPACING " << sx << " " << sy << " " << sz << "\n";
    out << "POINT_DATA " << static_cast<long long>(nxTot) * nyTot * nzTot << "\n";
    out << "SCALARS VOF float 1\n";
    out << "LOOKUP_TABLE default\n";
    return out.str();
}

// Values n0 .. n1 of the field as the reference's `out << value << "\n"` with
// setprecision(8) prints them: printf("%.8g") of the value widened to double.
void format_values(const float* f, size_t n0, size_t n1, std::string& out) {
    out.clear();
    out.reserve((n1 - n0) * 16);
    char buf[32];
    for (size_t q = n0; q < n1; ++q) {
        const auto r = std::to_chars(buf, buf + sizeof(buf), static_cast<double>(f[q]), std::chars_format::general, 8);
        out.append(buf, r.ptr);
        out.push_back('\n');
    }
}

bool write_vtk(const std::string& path, const float* f, int nxTot, int nyTot, int nzTot, Vtk kind,
               int threads) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const std::string head = vtk_header(nxTot, nyTot, nzTot, kind == Vtk::Binary);
    bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
    const size_t n = (size_t)nxTot * nyTot * nzTot;
    if (kind == Vtk::Binary) {
        std::vector<uint32_t> be(n);
        for (size_t q = 0; q < n; ++q) {
            uint32_t b;
            std::memcpy(&b, f + q, 4);
            be[q] = __builtin_bswap32(b);
        }
        ok = ok && std::fwrite(be.data(), 4, n, fp) == n;
        // legacy VTK binary data is followed by a newline
        ok = ok && std::fputc('\n', fp) != EOF;
    } else {
        // format chunks in parallel, write them in order
        const int nt = std::max(1, threads);
        const size_t chunk = (n + nt - 1) / nt;
        std::vector<std::string> parts(nt);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                const size_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
                format_values(f, a, b, parts[t]);
            });
        for (auto& th : pool) th.join();
        for (const auto& s : parts) ok = ok && std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    }
    return std::fclose(fp) == 0 && ok;
}

// Dumps of F taken off the solver's stream.
class Dumper {
  public:
    Dumper(vof_ctx* ctx, cudaStream_t solver, const vof_params& p, std::string dir, Vtk kind, int threads)
        : ctx_(ctx), solver_(solver), dir_(std::move(dir)), kind_(kind), threads_(threads), nxT_(p.nx + 2),
          nyT_(p.ny + 2), nzT_(p.nz + 2), n_((size_t)nxT_ * nyT_ * nzT_) {}

    int init() {
        if (kind_ == Vtk::None) return 0;
        if (cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking) != cudaSuccess) return -1;
        for (int b = 0; b < 2; ++b) {
            if (cudaMalloc(&stage_[b], n_ * sizeof(float)) != cudaSuccess) return -1;
            if (cudaMallocHost(&host_[b], n_ * sizeof(float)) != cudaSuccess) return -1;
            if (cudaEventCreateWithFlags(&staged_[b], cudaEventDisableTiming) != cudaSuccess) return -1;
            if (cudaEventCreateWithFlags(&landed_[b], cudaEventDisableTiming) != cudaSuccess) return -1;
            busy_[b] = false;
            used_[b] = false;
        }
        writer_ = std::thread([this] { run(); });
        return 0;
    }

    // Enqueue a dump of the current F for step istep (after the solver's
    // queued work); blocks only while both buffers are still being written.
    int dump(int istep) {
        if (kind_ == Vtk::None) return 0;
        int b;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_free_.wait(lk, [this] { return !busy_[0] || !busy_[1] || failed_; });
            if (failed_) return -1;
            b = !busy_[next_] ? next_ : next_ ^ 1;
            busy_[b] = true;
        }
        next_ = b ^ 1;
        // the staging buffer's previous copy to the host must be done first
        if (used_[b] && cudaStreamWaitEvent(solver_, landed_[b], 0) != cudaSuccess) return -1;
        used_[b] = true;
        if (vof_download(ctx_, VOF_FIELD_F, stage_[b], 1) != VOF_OK) return -1;
        if (cudaEventRecord(staged_[b], solver_) != cudaSuccess ||
            cudaStreamWaitEvent(side_, staged_[b], 0) != cudaSuccess ||
            cudaMemcpyAsync(host_[b], stage_[b], n_ * sizeof(float), cudaMemcpyDeviceToHost, side_) != cudaSuccess ||
            cudaEventRecord(landed_[b], side_) != cudaSuccess)
            return -1;
        {
            std::lock_guard<std::mutex> lk(mu_);
            jobs_.push_back({b, istep});
        }
        cv_job_.notify_one();
        return 0;
    }

    // Wait for every queued file; false if one could not be written.
    bool finish() {
        if (kind_ == Vtk::None) return true;
        {
            std::lock_guard<std::mutex> lk(mu_);
            done_ = true;
        }
        cv_job_.notify_one();
        if (writer_.joinable()) writer_.join();
        return !failed_;
    }

    ~Dumper() {
        finish();
        for (int b = 0; b < 2; ++b) {
            if (stage_[b]) cudaFree(stage_[b]);
            if (host_[b]) cudaFreeHost(host_[b]);
            if (staged_[b]) cudaEventDestroy(staged_[b]);
            if (landed_[b]) cudaEventDestroy(landed_[b]);
        }
        if (side_) cudaStreamDestroy(side_);
    }

  private:
    struct Job {
        int b, istep;
    };

    void run() {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_job_.wait(lk, [this] { return !jobs_.empty() || done_; });
                if (jobs_.empty()) return;
                j = jobs_.front();
                jobs_.pop_front();
            }
            bool ok = cudaEventSynchronize(landed_[j.b]) == cudaSuccess;
            std::ostringstream name;
            name << dir_ << "/step-" << std::setw(5) << std::setfill('0') << j.istep << ".vtk";
            ok = ok && write_vtk(name.str(), host_[j.b], nxT_, nyT_, nzT_, kind_, threads_);
            {
                std::lock_guard<std::mutex> lk(mu_);
                busy_[j.b] = false;
                if (!ok) failed_ = true;
            }
            if (!ok) std::cerr << "Failed to write output file: " << name.str() << std::endl;
            cv_free_.notify_all();
        }
    }

    vof_ctx* ctx_;
    cudaStream_t solver_, side_ = nullptr;
    std::string dir_;
    Vtk kind_;
    int threads_;
    int nxT_, nyT_, nzT_;
    size_t n_;
    float* stage_[2] = {nullptr, nullptr};
    float* host_[2] = {nullptr, nullptr};
    cudaEvent_t staged_[2] = {nullptr, nullptr}, landed_[2] = {nullptr, nullptr};
    bool busy_[2] = {false, false}, used_[2] = {false, false};
    int next_ = 0;
    bool done_ = false, failed_ = false;
    std::deque<Job> jobs_;
    std::mutex mu_;
    std::condition_variable cv_job_, cv_free_;
    std::thread writer_;
};

struct Options {
    int ic = 1, nstep = 100, max_steps = 0;
    int nx = 200, ny = 200, nz = 200;
    float gx = 0.0f, gy = -5.0f, gz = 0.0f, dt = 4.0e-6f;
    int jacobi = 10, mode = VOF_MODE_PLAIN;
    std::string out = "output", ic_file, final_prefix;
    Vtk vtk = Vtk::Ascii;
    int threads = 0;
    bool ic_only = false;
    float sigma = -1.0f;  // < 0: no surface-tension term (the reference's step)
};

void usage() {
    std::cout << "Usage: vof_drive [-ic 1|2|3] [--nstep N] [--max_steps N] [options]\n"
              << "  -ic         Initial condition selector. Only 1 is implemented, exactly as in the source.\n"
              << "  --nstep     Dump interval.\n"
              << "  --max_steps Number of steps to run. 0 means run until Ctrl+C.\n"
              << "Additions (the reference hardcodes these):\n"
              << "  --grid NX NY NZ      grid cells (default 200 200 200)\n"
              << "  --g GX GY GZ         gravity (default 0 -5 0)\n"
              << "  --dt DT              time step (default 4e-6)\n"
              << "  --jacobi N           Jacobi sweeps per step in plain mode (default 10)\n"
              << "  --mode M             plain | mixed | fp64 (default plain)\n"
              << "  --surface-tension S  add the continuum-surface-force term with sigma S (N/m)\n"
              << "  --out DIR            dump directory (default output)\n"
              << "  --vtk K              ascii (the reference's format) | binary | none\n"
              << "  --threads N          formatting threads for ASCII dumps (default: hardware)\n"
              << "  --ic-file PATH       initial F from raw float32, reference layout (replaces -ic)\n"
              << "  --final PREFIX       write PREFIX{F,U,V,W,P}.raw (float32, reference layout) at the end\n"
              << "  --ic-only            write the initial F as step-00000.vtk and exit (no GPU work)\n";
}

int parse(int argc, char** argv, Options& o) {
    for (int a = 1; a < argc; ++a) {
        const std::string arg = argv[a];
        auto need = [&](int k) { return a + k < argc; };
        if (arg == "-ic" && need(1)) o.ic = std::atoi(argv[++a]);
        else if (arg == "--nstep" && need(1)) o.nstep = std::atoi(argv[++a]);
        else if (arg == "--max_steps" && need(1)) o.max_steps = std::atoi(argv[++a]);
        else if (arg == "--grid" && need(3)) {
            o.nx = std::atoi(argv[++a]);
            o.ny = std::atoi(argv[++a]);
            o.nz = std::atoi(argv[++a]);
        } else if (arg == "--g" && need(3)) {
            o.gx = std::strtof(argv[++a], nullptr);
            o.gy = std::strtof(argv[++a], nullptr);
            o.gz = std::strtof(argv[++a], nullptr);
        } else if (arg == "--dt" && need(1)) o.dt = std::strtof(argv[++a], nullptr);
        else if (arg == "--jacobi" && need(1)) o.jacobi = std::atoi(argv[++a]);
        else if (arg == "--mode" && need(1)) {
            const std::string m = argv[++a];
            if (m == "plain") o.mode = VOF_MODE_PLAIN;
            else if (m == "mixed") o.mode = VOF_MODE_MIXED;
            else if (m == "fp64") o.mode = VOF_MODE_FP64;
            else return -1;
        } else if (arg == "--surface-tension" && need(1)) {
            o.sigma = std::strtof(argv[++a], nullptr);
            if (!(o.sigma >= 0.0f)) return -1;
        } else if (arg == "--out" && need(1)) o.out = argv[++a];
        else if (arg == "--vtk" && need(1)) {
            const std::string k = argv[++a];
            if (k == "ascii") o.vtk = Vtk::Ascii;
            else if (k == "binary") o.vtk = Vtk::Binary;
            else if (k == "none") o.vtk = Vtk::None;
            else return -1;
        } else if (arg == "--threads" && need(1)) o.threads = std::atoi(argv[++a]);
        else if (arg == "--ic-file" && need(1)) o.ic_file = argv[++a];
        else if (arg == "--final" && need(1)) o.final_prefix = argv[++a];
        else if (arg == "--ic-only") o.ic_only = true;
        else if (arg == "--help" || arg == "-h") return 1;
        else {
            std::cerr << "Unknown argument: " << arg << std::endl;
            return -1;
        }
    }
    return 0;
}

bool read_raw(const std::string& path, std::vector<float>& v, size_t n) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    v.resize(n);
    const bool ok = std::fread(v.data(), sizeof(float), n, fp) == n;
    std::fclose(fp);
    return ok;
}

bool write_raw(const std::string& path, const std::vector<float>& v) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(v.data(), sizeof(float), v.size(), fp) == v.size();
    return std::fclose(fp) == 0 && ok;
}

int fail(const char* what, int st, vof_ctx* ctx) {
    std::cerr << what << " failed: " << vof_error_string(st);
    if (ctx && st == VOF_E_CUDA) std::cerr << " (" << cudaGetErrorString((cudaError_t)vof_last_cuda_error(ctx)) << ")";
    std::cerr << std::endl;
    return EXIT_FAILURE;
}

}  // namespace

int main(int argc, char** argv) {
    std::signal(SIGINT, handle_signal);
    Options o;
    const int pr = parse(argc, argv, o);
    if (pr == 1) {
        usage();
        return 0;
    }
    if (pr < 0) {
        usage();
        return EXIT_FAILURE;
    }
    if (o.ic < 1 || o.ic > 3) {
        std::cerr << "Invalid initial condition. Allowed values: 1, 2, 3" << std::endl;
        return EXIT_FAILURE;
    }
    if (o.nstep < 1) {
        std::cerr << "--nstep must be at least 1" << std::endl;
        return EXIT_FAILURE;
    }
    if (o.threads <= 0) o.threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));

    vof_params p;
    int st = vof_params_init(&p, o.nx, o.ny, o.nz);
    if (st != VOF_OK) return fail("vof_params_init", st, nullptr);
    p.gx = o.gx;
    p.gy = o.gy;
    p.gz = o.gz;
    p.dt = o.dt;
    p.jacobi_iters = o.jacobi;
    p.mode = o.mode;
    if (o.sigma >= 0.0f) {
        p.sigma = o.sigma;
        p.surface_tension = 1;
    }
    if ((st = vof_params_finalize(&p)) != VOF_OK) return fail("vof_params_finalize", st, nullptr);

    // the initial F in the reference layout, then apply_bc_F once (voftrial1.cu:1334-1337)
    const size_t ntot = (size_t)p.nTot;
    std::vector<float> F;
    if (!o.ic_file.empty()) {
        if (!read_raw(o.ic_file, F, ntot)) {
            std::cerr << "Failed to read " << o.ic_file << std::endl;
            return EXIT_FAILURE;
        }
    } else {
        init_F(p, o.ic, F);
    }
    bc_F(p, F);
    mkdir(o.out.c_str(), 0755);  // std::system("mkdir -p output") in the reference
    if (o.ic_only) {
        const bool ok = o.vtk == Vtk::None ||
                        write_vtk(o.out + "/step-00000.vtk", F.data(), p.nx + 2, p.ny + 2, p.nz + 2, o.vtk, o.threads);
        return ok ? 0 : EXIT_FAILURE;
    }

    std::cout << ">>> A 3D VOF solver ported to CUDA (speed-tuned path)\n";
    std::cout << ">>> Grid resolution: " << p.nx << " x " << p.ny << " x " << p.nz << ", dt = " << std::scientific
              << p.dt << std::defaultfloat << "\n";
    std::cout << ">>> Density ratio: " << (p.rho_l / p.rho_g) << ", gravity : " << p.gy << ", sigma : " << p.sigma
              << "\n";
    std::cout << ">>> Viscosity ratio: " << (p.nu_l / p.nu_g) << "\n";

    cudaStream_t stream = nullptr;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
        std::cerr << "cudaStreamCreate failed" << std::endl;
        return EXIT_FAILURE;
    }
    vof_ctx* ctx = nullptr;
    if ((st = vof_create(&p, stream, &ctx)) != VOF_OK) return fail("vof_create", st, nullptr);
    if ((st = vof_upload(ctx, VOF_FIELD_F, F.data(), 0)) != VOF_OK || (st = vof_sync(ctx)) != VOF_OK)
        return fail("vof_upload", st, ctx);

    int rc = 0;
    int istep = 0;
    {
        Dumper dumper(ctx, stream, p, o.out, o.vtk, o.threads);
        if (dumper.init() != 0) {
            std::cerr << "Failed to set up the output buffers" << std::endl;
            vof_destroy(ctx);
            return EXIT_FAILURE;
        }
        auto t0 = std::chrono::steady_clock::now();
        // steps between dumps in graph-captured batches; Ctrl+C is checked
        // between batches of at most 64 steps
        while (!g_stop && (o.max_steps == 0 || istep < o.max_steps)) {
            int n = o.nstep - istep % o.nstep;
            if (o.max_steps > 0) n = std::min(n, o.max_steps - istep);
            n = std::min(n, 64);
            st = vof_run(ctx, istep + 1, n);
            if (st == VOF_E_NOT_CONVERGED) {  // convergent modes: a solve hit max_outer; keep going
                std::cerr << ">>> Warning: a pressure solve in steps " << istep + 1 << ".." << istep + n
                          << " stopped at max_outer before tol" << std::endl;
            } else if (st != VOF_OK) {
                rc = fail("vof_run", st, ctx);
                break;
            }
            istep += n;
            if (istep % o.nstep == 0) {
                std::cout << ">>> Exporting step-" << std::setw(5) << std::setfill('0') << istep << " result..."
                          << std::setfill(' ') << std::endl;
                if (dumper.dump(istep) != 0) {
                    std::cerr << "Dump of step " << istep << " failed" << std::endl;
                    rc = EXIT_FAILURE;
                    break;
                }
            }
        }
        if ((st = vof_sync(ctx)) != VOF_OK && rc == 0) rc = fail("vof_sync", st, ctx);
        if (!dumper.finish()) rc = EXIT_FAILURE;
        auto t1 = std::chrono::steady_clock::now();
        const double elapsed = std::chrono::duration_cast<std::chrono::duration<double>>(t1 - t0).count();
        std::cout << ">>> Finished at step " << istep << " in " << elapsed << " s" << std::endl;
    }
    if (rc == 0 && !o.final_prefix.empty()) {
        static const char* names[5] = {"F", "U", "V", "W", "P"};
        std::vector<float> buf(ntot);
        for (int f = 0; f < 5 && rc == 0; ++f) {
            if ((st = vof_download(ctx, f, buf.data(), 0)) != VOF_OK) rc = fail("vof_download", st, ctx);
            else if (!write_raw(o.final_prefix + names[f] + ".raw", buf)) {
                std::cerr << "Failed to write " << o.final_prefix << names[f] << ".raw" << std::endl;
                rc = EXIT_FAILURE;
            }
        }
    }
    vof_destroy(ctx);
    cudaStreamDestroy(stream);
    return rc;
}
