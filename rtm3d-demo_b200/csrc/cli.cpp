// cli.cpp -- rtm3d_b200: the command-line host of librtm3d_b200.
//
//   rtm3d_b200 input.json
//
// Reads the reference's input.json unchanged (all keys of RTMParam, include/RTMParam.hpp:115-186,
// with the same types, plus "verbose"), and runs the same process as the reference program
// (src/Main.cpp:11-48 -> RTMAcousticProcess::rtm, src/process/RTMAcousticProcess.cpp:8-60):
//   modeling   one shot record per shot, written as .seism chunks of ntstep steps into datdir
//              (by a background task, while the next shot runs)
//              (RTMAcousticController::rtmDistShotModeling, src/controller/RTMAcousticController.cpp:129-170);
//   migration  .seism chunks read back per shot (the next shot's by a background task while this
//              one runs), HBC or RBC migration, images stacked, order-2
//              Laplacian filter, borders removed, RTMIMG file written into outdir
//              (rtmDistShotMigration, :172-269).
// Velocity preparation follows RTMController::loadRTMVelocitiesModel (src/controller/RTMController.cpp:27-119):
// extend the borders, ABC border for modeling, the migration border otherwise (or the extended
// model from vpefile), optional save of the extended model, then v^2 dt^2.
//
// Optional keys the reference does not read (its validation ignores unknown keys):
//   "b200_fast_fma" (bool)   FMA form of the stencil (not bit-exact with the reference CPU path)
//   "b200_device"   (uint)   CUDA device ordinal
//   "b200_rbc_seed" (uint)   seed of the random border (libc srand; the reference leaves rand() unseeded)
//   fmig       frequency-domain migration instead (RTMFreqDomainKernel, selected by "fmig": true,
//              src/process/RTMAcousticProcess.cpp:16-18), fmig_nwstep frequencies per pass over
//              time as the reference's accelerator builds take it (0: all in one pass, the CPU
//              build's order).
// 2D models (nx == 1) run the reference's 2D step (the plane x = blen, no x term).
// Out of scope and rejected: distributed_grid and fmig_distributed_imaging (MPI partitions).
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <future>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "json.hpp"
#include "rtm3d_b200.h"

namespace {

using rtmbjson::Kind;
using rtmbjson::Value;

struct Param {
    std::string mname, vpfile, vpefile, outdir, tmpdir, datdir, rtm_type, boundary_condition;
    unsigned nx, ny, nz, blen, nt, stencil_order, ntstep, nthreads, snapshot_step;
    unsigned source_start_x, source_start_y, source_depth_z, source_distance_x, source_distance_y;
    unsigned source_count_x, source_count_y;
    unsigned receiver_start_x, receiver_start_y, receiver_depth_z, receiver_distance_x, receiver_distance_y;
    unsigned receiver_count_x, receiver_count_y;
    float dx, dy, dz, dt, fpeak, taper_factor;
    bool modeling, migration, save_vpe_file, load_vpe_from_file, verbose, save_snapshots, distributed_grid, fmig;
    bool fmig_distributed_imaging;
    float fmig_min_freq, fmig_max_freq;
    unsigned fmig_nwstep;
    bool fast_fma = false;
    int device = -1;
    long long rbc_seed = -1;
};

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void say(const Param &p, const std::string &msg) {
    if (p.verbose) std::cout << "> " << msg << std::endl;
}

// RTMParam::validateParameters (src/param/RTMParam.cpp:59-96): every listed key present with the
// listed JSON type.
void validate(const Value &root) {
    static const std::vector<std::pair<const char *, Kind>> keys = {
        {"mname", Kind::String}, {"vpfile", Kind::String}, {"vpefile", Kind::String},
        {"save_vpe_file", Kind::Bool}, {"outdir", Kind::String}, {"tmpdir", Kind::String},
        {"datdir", Kind::String}, {"nx", Kind::Unsigned}, {"ny", Kind::Unsigned}, {"nz", Kind::Unsigned},
        {"blen", Kind::Unsigned}, {"width_m", Kind::Unsigned}, {"height_m", Kind::Unsigned},
        {"depth_m", Kind::Unsigned}, {"nt", Kind::Unsigned}, {"dz", Kind::Float}, {"dy", Kind::Float},
        {"dx", Kind::Float}, {"dt", Kind::Float}, {"fpeak", Kind::Float}, {"fmax", Kind::Float},
        {"taper_factor", Kind::Float}, {"stencil_order", Kind::Unsigned}, {"modeling", Kind::Bool},
        {"migration", Kind::Bool}, {"rtm_type", Kind::String}, {"boundary_condition", Kind::String},
        {"source_total", Kind::Unsigned}, {"source_start_x", Kind::Unsigned}, {"source_start_y", Kind::Unsigned},
        {"source_depth_z", Kind::Unsigned}, {"source_distance_x", Kind::Unsigned},
        {"source_distance_y", Kind::Unsigned}, {"source_count_x", Kind::Unsigned},
        {"source_count_y", Kind::Unsigned}, {"receiver_total", Kind::Unsigned},
        {"receiver_start_x", Kind::Unsigned}, {"receiver_start_y", Kind::Unsigned},
        {"receiver_depth_z", Kind::Unsigned}, {"receiver_distance_x", Kind::Unsigned},
        {"receiver_distance_y", Kind::Unsigned}, {"receiver_count_x", Kind::Unsigned},
        {"receiver_count_y", Kind::Unsigned}, {"ntstep", Kind::Unsigned}, {"nthreads", Kind::Unsigned},
        {"load_vpe_from_file", Kind::Bool}, {"save_snapshots", Kind::Bool}, {"distributed_grid", Kind::Bool},
        {"snapshot_step", Kind::Unsigned}, {"fmig", Kind::Bool}, {"fmig_max_freq", Kind::Float},
        {"fmig_min_freq", Kind::Float}, {"fmig_nwstep", Kind::Unsigned}, {"fmig_distributed_imaging", Kind::Bool},
        {"fpga_xclbin", Kind::String}, {"fpga_fwd_kernel", Kind::String}, {"fpga_bwd_kernel", Kind::String},
        {"verbose", Kind::Bool}};
    if (root.kind != Kind::Object) throw Error("[ input.json must hold a JSON object ]");
    for (const auto &k : keys) {
        auto it = root.obj.find(k.first);
        const Kind got = it == root.obj.end() ? Kind::Null : it->second.kind;
        if (got != k.second)
            throw Error(std::string("[ Input parameter '") + k.first + "' has wrong type! Expected: '" +
                        rtmbjson::kind_name(k.second) + "' got: '" + rtmbjson::kind_name(got) + "' ]");
    }
}

Param load_param(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw Error("[ Input File '" + path + "' doesn't exists. Please check input file path. ]");
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    Value root = rtmbjson::Parser(text).parse();
    validate(root);
    auto &o = root.obj;
    auto U = [&](const char *k) { return static_cast<unsigned>(o.at(k).u); };
    auto F = [&](const char *k) { return static_cast<float>(o.at(k).num); };
    auto B = [&](const char *k) { return o.at(k).b; };
    auto S = [&](const char *k) { return o.at(k).s; };
    Param p;
    p.mname = S("mname"); p.vpfile = S("vpfile"); p.vpefile = S("vpefile"); p.outdir = S("outdir");
    p.tmpdir = S("tmpdir"); p.datdir = S("datdir"); p.rtm_type = S("rtm_type");
    p.boundary_condition = S("boundary_condition");
    p.nx = U("nx"); p.ny = U("ny"); p.nz = U("nz"); p.blen = U("blen"); p.nt = U("nt");
    p.stencil_order = U("stencil_order"); p.ntstep = U("ntstep"); p.nthreads = U("nthreads");
    p.snapshot_step = U("snapshot_step");
    p.source_start_x = U("source_start_x"); p.source_start_y = U("source_start_y");
    p.source_depth_z = U("source_depth_z"); p.source_distance_x = U("source_distance_x");
    p.source_distance_y = U("source_distance_y"); p.source_count_x = U("source_count_x");
    p.source_count_y = U("source_count_y");
    p.receiver_start_x = U("receiver_start_x"); p.receiver_start_y = U("receiver_start_y");
    p.receiver_depth_z = U("receiver_depth_z"); p.receiver_distance_x = U("receiver_distance_x");
    p.receiver_distance_y = U("receiver_distance_y"); p.receiver_count_x = U("receiver_count_x");
    p.receiver_count_y = U("receiver_count_y");
    p.dx = F("dx"); p.dy = F("dy"); p.dz = F("dz"); p.dt = F("dt"); p.fpeak = F("fpeak");
    p.taper_factor = F("taper_factor");
    p.modeling = B("modeling"); p.migration = B("migration"); p.save_vpe_file = B("save_vpe_file");
    p.load_vpe_from_file = B("load_vpe_from_file"); p.verbose = B("verbose");
    p.save_snapshots = B("save_snapshots"); p.distributed_grid = B("distributed_grid"); p.fmig = B("fmig");
    p.fmig_distributed_imaging = B("fmig_distributed_imaging");
    p.fmig_min_freq = F("fmig_min_freq"); p.fmig_max_freq = F("fmig_max_freq"); p.fmig_nwstep = U("fmig_nwstep");
    if (o.count("b200_fast_fma") && o.at("b200_fast_fma").kind == Kind::Bool) p.fast_fma = o.at("b200_fast_fma").b;
    if (o.count("b200_device") && o.at("b200_device").kind == Kind::Unsigned) p.device = (int)o.at("b200_device").u;
    if (o.count("b200_rbc_seed") && o.at("b200_rbc_seed").kind == Kind::Unsigned)
        p.rbc_seed = (long long)o.at("b200_rbc_seed").u;
    // RTMParam::loadRTMParam (:241-245)
    if (p.nt < p.ntstep) throw Error("[ RTMParam Error: NT smaller than NTSTEP ]");
    if (p.ntstep == 0 || p.nt % p.ntstep) throw Error("[ nt must be a multiple of ntstep ]");
    if (p.fmig && p.fmig_max_freq <= p.fmig_min_freq)  // RTMParam.cpp:246-251
        throw Error("[ RTMParam Error: fmig_max_freq must be greater than fmig_min_freq ]");
    if (p.fmig && p.fmig_distributed_imaging)
        throw Error("[ fmig_distributed_imaging (MPI partition of the image) is not supported: one GPU holds the volume ]");
    if (p.distributed_grid) throw Error("[ distributed_grid (MPI halo decomposition) is not supported: one GPU holds the volume ]");
    return p;
}

std::vector<float> read_floats(const std::string &path, size_t n) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Error("Input grid file '" + path + "' doesn't exist! Please check.");
    std::vector<float> v(n);
    f.read(reinterpret_cast<char *>(v.data()), n * sizeof(float));
    if (static_cast<size_t>(f.gcount()) != n * sizeof(float))
        throw Error("Input grid file '" + path + "' is shorter than expected");
    return v;
}

void write_floats(const std::string &path, const float *v, size_t n) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw Error("Output grid file '" + path + "' could not be opened.");
    f.write(reinterpret_cast<const char *>(v), n * sizeof(float));
    if (!f) throw Error("Output grid file '" + path + "' could not be written.");
}

// include/RTMBase.hpp:131-138
std::string seismogram_name(const Param &p, int sx, int sy, int sz, unsigned itstart) {
    return p.datdir + "/RTMSEISMOGRAM_S" + std::to_string(sx) + "x" + std::to_string(sy) + "x" +
           std::to_string(sz) + "_NXNY_" + std::to_string(p.receiver_count_x) + "x" +
           std::to_string(p.receiver_count_y) + "_NTSTART" + std::to_string(itstart) + "_NTSTEP" +
           std::to_string(p.ntstep) + ".seism";
}

// include/RTMBase.hpp:79-91 (single process: NP1)
std::string image_name(const Param &p, unsigned nshots) {
    std::string m = p.mname;
    std::transform(m.begin(), m.end(), m.begin(), [](unsigned char c) { return std::toupper(c); });
    return p.outdir + "/RTMIMG_" + m + "_NS" + std::to_string(nshots) + "_NXNYNZ_" + std::to_string(p.nx) + "x" +
           std::to_string(p.ny) + "x" + std::to_string(p.nz) + "_NT" + std::to_string(p.nt) + ".bin.NP1";
}

int bc_code(const std::string &s) {  // getRTMBoundaryCondition (include/RTMGrid.hpp:39-57)
    if (s == "rbc") return RTMB_BC_RBC;
    if (s == "abc") return RTMB_BC_ABC;
    return RTMB_BC_HBC;
}

void check(int rc, rtmb_ctx *ctx, const char *what) {
    if (rc != RTMB_OK)
        throw Error(std::string(what) + " failed (" + std::to_string(rc) + "): " + (ctx ? rtmb_last_error(ctx) : ""));
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int run(const Param &p) {
    const size_t nxe = p.nx + 2 * p.blen, nye = p.ny + 2 * p.blen, nze = p.nz + 2 * p.blen;
    const size_t n = nxe * nye * nze;
    say(p, "Loading velocity model '" + p.mname + "' from '" + p.vpfile + "'");
    std::vector<float> v = read_floats(p.vpfile, (size_t)p.nx * p.ny * p.nz);
    std::vector<float> ve(n);
    const bool mig = !p.modeling && p.migration;
    const int bc = p.modeling ? RTMB_BC_ABC : bc_code(p.boundary_condition);  // modeling always uses ABC
    check(rtmb_prepare_velocity(v.data(), p.nx, p.ny, p.nz, p.blen, bc, p.rbc_seed, ve.data()), nullptr,
          "velocity border initialisation");
    if (mig && p.load_vpe_from_file) {
        say(p, "Loading extended velocity model from '" + p.vpefile + "'");
        ve = read_floats(p.vpefile, n);
    }
    if (p.save_vpe_file) write_floats(p.vpefile, ve.data(), n);
    check(rtmb_v2dt2_host(ve.data(), n, p.dt), nullptr, "v2dt2");

    rtmb_params rp{};
    rp.nx = p.nx; rp.ny = p.ny; rp.nz = p.nz; rp.blen = p.blen; rp.nt = p.nt; rp.ntstep = p.ntstep;
    rp.stencil_order = p.stencil_order; rp.dx = p.dx; rp.dy = p.dy; rp.dz = p.dz; rp.dt = p.dt;
    rp.fpeak = p.fpeak; rp.taper_factor = p.taper_factor;
    rp.receiver_start_x = p.receiver_start_x; rp.receiver_start_y = p.receiver_start_y;
    rp.receiver_depth_z = p.receiver_depth_z; rp.receiver_distance_x = p.receiver_distance_x;
    rp.receiver_distance_y = p.receiver_distance_y; rp.receiver_count_x = p.receiver_count_x;
    rp.receiver_count_y = p.receiver_count_y; rp.boundary = bc; rp.flags = p.fast_fma ? RTMB_FLAG_FAST_FMA : 0u;
    rp.device = p.device;
    rtmb_ctx *ctx = nullptr;
    check(rtmb_create(&rp, &ctx), nullptr, "rtmb_create");
    struct Guard { rtmb_ctx *c; ~Guard() { rtmb_destroy(c); } } guard{ctx};
    check(rtmb_load_v2dt2(ctx, ve.data(), 1), ctx, "rtmb_load_v2dt2");
    ve.clear(); ve.shrink_to_fit();

    const size_t chunk = (size_t)p.receiver_count_x * p.receiver_count_y * p.ntstep;
    const size_t nchunks = p.nt / p.ntstep;
    const size_t nrec = chunk * nchunks;
    float *d_rec = nullptr, *d_img = nullptr, *d_stack = nullptr, *d_out = nullptr;
    struct DevFree { float **ps[4]; ~DevFree() { for (auto p : ps) if (*p) cudaFree(*p); } } dfree{{&d_rec, &d_img, &d_stack, &d_out}};
    // two pinned host records: the shot being computed and the one being read (migration) or
    // written (modeling) by the I/O thread at the same time
    float *h_rec[2] = {nullptr, nullptr};
    struct HostFree { float **ps[2]; ~HostFree() { for (auto p : ps) if (*p) cudaFreeHost(*p); } } hfree{{&h_rec[0], &h_rec[1]}};
    for (auto &h : h_rec)
        if (cudaMallocHost(&h, std::max<size_t>(nrec, 1) * sizeof(float)) != cudaSuccess)
            throw Error("pinned host allocation failed");
    const unsigned nshots = p.source_count_x * p.source_count_y;
    double t_total = 0.0;
    if (mig) {
        if (cudaMalloc(&d_rec, std::max<size_t>(nrec, 1) * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&d_img, n * sizeof(float)) != cudaSuccess || cudaMalloc(&d_stack, n * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&d_out, (size_t)p.nx * p.ny * p.nz * sizeof(float)) != cudaSuccess ||
            cudaMemset(d_stack, 0, n * sizeof(float)) != cudaSuccess)
            throw Error("device allocation failed");
    }
    // the shots in the reference's order (RTMController.cpp:139-165)
    struct Shot { unsigned sx, sy, sz; };
    std::vector<Shot> shots;
    for (unsigned ix = 0; ix < p.source_count_x; ++ix)
        for (unsigned iy = 0; iy < p.source_count_y; ++iy) {
            const Shot s{ix * p.source_distance_x + p.source_start_x, iy * p.source_distance_y + p.source_start_y,
                         p.source_depth_z};
            if (s.sx >= p.nx || s.sy >= p.ny || s.sz >= p.nz)
                throw Error("[ Invalid Source Position: (" + std::to_string(s.sx) + "," + std::to_string(s.sy) + "," +
                            std::to_string(s.sz) + ") ]");
            shots.push_back(s);
        }
    // record I/O off the compute path: one background task at a time reads the next shot's
    // .seism chunks (migration) or writes the previous shot's (modeling) while the GPU runs
    auto read_record = [&](const Shot &s, float *dst) {
        for (size_t c = 0; c < nchunks; ++c) {
            std::ifstream f(seismogram_name(p, s.sx, s.sy, s.sz, (unsigned)(c * p.ntstep)), std::ios::binary);
            if (!f) throw Error("Input grid file '" + seismogram_name(p, s.sx, s.sy, s.sz, (unsigned)(c * p.ntstep)) +
                                "' doesn't exist! Please check.");
            f.read(reinterpret_cast<char *>(dst + c * chunk), chunk * sizeof(float));
            if (static_cast<size_t>(f.gcount()) != chunk * sizeof(float)) throw Error("seismogram file too short");
        }
    };
    auto write_record = [&](const Shot &s, const float *src) {
        for (size_t c = 0; c < nchunks; ++c)
            write_floats(seismogram_name(p, s.sx, s.sy, s.sz, (unsigned)(c * p.ntstep)), src + c * chunk, chunk);
    };
    std::future<void> io, wr[2];  // io: the reader; wr[b]: the writer of host buffer b
    if (mig && !shots.empty()) io = std::async(std::launch::async, read_record, shots[0], h_rec[0]);
    for (size_t k = 0; k < shots.size(); ++k) {
        const Shot &s = shots[k];
        say(p, "Shot " + std::to_string(k + 1) + "/" + std::to_string(nshots) + " (" + std::to_string(s.sx) + "," +
                   std::to_string(s.sy) + "," + std::to_string(s.sz) + "):");
        float *rec = h_rec[k & 1];
        if (p.modeling) {
            // buffer k & 1 may still be written out for shot k-2; shot k-1's files are written
            // meanwhile from the other buffer while this shot runs
            if (wr[k & 1].valid()) wr[k & 1].get();
            const auto t0 = std::chrono::steady_clock::now();
            check(rtmb_model_shot_host(ctx, s.sx, s.sy, s.sz, rec), ctx, "modeling");
            t_total += seconds_since(t0);
            wr[k & 1] = std::async(std::launch::async, write_record, s, rec);
        } else if (mig) {
            io.get();  // this shot's record is on the host
            if (k + 1 < shots.size()) io = std::async(std::launch::async, read_record, shots[k + 1], h_rec[(k + 1) & 1]);
            const auto t0 = std::chrono::steady_clock::now();
            if (cudaMemcpy(d_rec, rec, nrec * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
                throw Error("record upload failed");
            if (p.fmig)
                check(rtmb_migrate_shot_fmig(ctx, s.sx, s.sy, s.sz, d_rec, p.fmig_min_freq, p.fmig_max_freq,
                                             p.fmig_nwstep, d_img),
                      ctx, "frequency-domain migration");
            else
                check(rtmb_migrate_shot(ctx, s.sx, s.sy, s.sz, d_rec, d_img), ctx, "migration");
            check(rtmb_image_stack(ctx, d_stack, d_img), ctx, "image stack");
            check(rtmb_sync(ctx), ctx, "sync");
            t_total += seconds_since(t0);
        }
    }
    if (io.valid()) io.get();
    for (auto &w : wr)
        if (w.valid()) w.get();
    if (mig) {
        check(rtmb_image_finalize(ctx, d_stack, d_out), ctx, "image filter");
        check(rtmb_sync(ctx), ctx, "sync");
        std::vector<float> img((size_t)p.nx * p.ny * p.nz);
        if (cudaMemcpy(img.data(), d_out, img.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw Error("image download failed");
        const std::string name = image_name(p, nshots);
        say(p, "Saving rtm output image at: " + name);
        write_floats(name, img.data(), img.size());
    }
    if (p.verbose) {
        double sweeps = p.modeling ? p.nt : (3.0 * p.nt - 2.0);
        if (p.fmig) {  // two wavefields stepped per pass over time, one pass per group of frequencies
            const int nw = rtmb_fmig_nw(p.dt, p.nt, p.fmig_min_freq, p.fmig_max_freq);
            const int nws = (p.fmig_nwstep == 0 || (int)p.fmig_nwstep > nw) ? nw : (int)p.fmig_nwstep;
            sweeps = 2.0 * p.nt * (nws > 0 ? (nw + nws - 1) / nws : 0);
        }
        const double pts = double(n) * sweeps * nshots;
        std::printf("{\n  \"mname\": %s\n  \"nx\":%u\n  \"ny\":%u\n  \"nz\":%u\n  \"nt\":%u\n  \"%s_time\":%f\n"
                    "  \"gpoint_updates_per_s\":%f\n}\n",
                    p.mname.c_str(), p.nx, p.ny, p.nz, p.nt, p.modeling ? "modeling" : "migration", t_total,
                    t_total > 0 ? pts / t_total / 1e9 : 0.0);
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        std::cout << "> You forgot the input.json file!" << std::endl;
        return -1;
    }
    try {
        Param p = load_param(argv[1]);
        return run(p);
    } catch (const std::exception &e) {
        std::cout << "> Error:\n" << e.what() << "\n> Aborting!" << std::endl;
        return 1;
    }
}
