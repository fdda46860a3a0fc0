// Header-only C++ shim that re-creates the iterNLM driver's classes on top of
// the C ABI in include/inlm.h, so a driver written against the reference keeps
// its flow: protocol::DenoiseParameters (denoise_parameters.h:9-84),
// denoise::IterativeNLM_GPU (Denoiser/iternlm_gpu.h:20-56), noise::NoiseLevel
// (Noise/noiselevel.h:17-45) and the TIFF / noise-file parts of
// hdcom::HdCommunication (Geometry/hdcommunication.h).
//
// Errors: the reference's void members report nothing; here each object keeps
// the status of its last call (`status`, 0 = OK) and prints the library's
// error text, and configure_device returns -1 without a GPU and -2 on a CUDA
// error as the reference does.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <filesystem>
#include <sys/stat.h>
#include <vector>

#include "inlm.h"

namespace protocol {

// Field names and defaults of the reference's parameter block; `seed` and
// `precision` are additions (the reference seeds its sampler with time()).
struct DenoiseParameters {
    float alpha = 0.5f;
    int maxiterations = 4;
    int nslices = 11;
    int radius_searchspace[3] = {10, 10, 10};
    int radius_patchspace[3] = {1, 1, 1};
    float beta = 1.f;
    float z_anisotropy = 1.f;

    struct NoiseLevel {
        std::string mode = "z-adaptive";  // "z-adaptive", "global", "manual", "semimanual"
        int zwindow = 100;
        float sigma[2] = {0.0f, 0.0f};
        uint64_t n_samples = 100000;
        int patchsize = 15;
        float stds_from_mean = 1;
        bool continuous_estimate = false;
        int circular_mask_diameter = 0;
        unsigned int seed = 0;  // 0: time(NULL), as NoiseLevel's constructor seeds rand()
    };
    struct CPU {
        int max_threads = 128;
        bool unrolled_patchspace = false;
        bool blockwise = true;
    };
    struct GPU {
        int n_gpus = 2;
        int deviceID = 0;
        int threadsPerBlock = 128;
        int memory_buffer = 0;
        bool blockwise_host = false;
        std::string precision = "f32";  // "f32" (bit-exact) or "f16" (FP16 storage form)
    };
    struct IO {
        bool resume = false;
        int firstslice = -1;
        int lastslice = -1;
        std::string save_type = "32bit";
        bool cleanup = false;
        bool rgb = false;
        std::string active_outpath = "";
    };
    struct Color {
        bool stabilize_variance = true;
        bool independent_channels = false;
        bool average_channelsigma = true;
    };

    NoiseLevel noiselevel;
    CPU cpu;
    GPU gpu;
    IO io;
    Color color;
};

inline int noise_mode_code(const std::string& m) {
    if (m == "global") return INLM_NOISE_GLOBAL;
    if (m == "manual") return INLM_NOISE_MANUAL;
    if (m == "semimanual") return INLM_NOISE_SEMIMANUAL;
    return INLM_NOISE_ZADAPTIVE;
}

inline inlm_params to_inlm(const DenoiseParameters& p) {
    inlm_params q;
    inlm_default_params(&q);
    q.alpha = p.alpha;
    q.maxiterations = p.maxiterations;
    q.nslices = p.nslices;
    for (int i = 0; i < 3; i++) {
        q.search_radius[i] = p.radius_searchspace[i];
        q.patch_radius[i] = p.radius_patchspace[i];
    }
    q.beta = p.beta;
    q.z_anisotropy = p.z_anisotropy;
    q.noise_mode = noise_mode_code(p.noiselevel.mode);
    q.zwindow = p.noiselevel.zwindow;
    q.sigma[0] = p.noiselevel.sigma[0];
    q.sigma[1] = p.noiselevel.sigma[1];
    q.n_samples = p.noiselevel.n_samples;
    q.noise_patchsize = p.noiselevel.patchsize;
    q.stds_from_mean = p.noiselevel.stds_from_mean;
    q.continuous_estimate = p.noiselevel.continuous_estimate ? 1 : 0;
    q.circular_mask_diameter = p.noiselevel.circular_mask_diameter;
    q.noise_seed = p.noiselevel.seed ? p.noiselevel.seed : (unsigned int)time(nullptr);
    q.device_id = p.gpu.deviceID;
    q.precision = p.gpu.precision == "f16" ? INLM_PRECISION_F16 : INLM_PRECISION_F32;
    return q;
}

inline int report(int rc, const char* where) {
    if (rc != INLM_OK) std::cout << "Error! " << where << ": " << inlm_last_error() << std::endl;
    return rc;
}

}  // namespace protocol

namespace hdcom {

inline std::string zfill_int2string(int v, unsigned int width) {
    std::string s = std::to_string(v);
    while (s.size() < width) s = "0" + s;
    return s;
}

// true when every slice file first..last of an iteration directory exists and
// all have one size (the --resume test, iternlm_gpu.cu:1665-1684)
inline bool iteration_on_disk(const std::string& dir, int first, int last) {
    long long size = -1;
    for (int i = first; i <= last; i++) {
        struct stat st;
        const std::string f = dir + "/denoised" + zfill_int2string(i, 4) + ".tif";
        if (stat(f.c_str(), &st) != 0) return false;
        if (size < 0) size = (long long)st.st_size;
        else if ((long long)st.st_size != size) return false;
    }
    return true;
}

// The slices first..last of an iteration directory (malloc'd), NULL on error.
inline float* read_iteration(const std::string& dir, int first, int last, int shape[3]) {
    const size_t nslice = (size_t)shape[0] * shape[1];
    float* out = (float*)malloc(nslice * shape[2] * sizeof(float));
    for (int i = first; i <= last; i++) {
        const std::string f = dir + "/denoised" + zfill_int2string(i, 4) + ".tif";
        if (inlm_tiff_read(f.c_str(), -1, -1, out + (size_t)(i - first) * nslice, nslice) != INLM_OK) {
            protocol::report(INLM_ERR_IO, "resume");
            free(out);
            return nullptr;
        }
    }
    return out;
}

}  // namespace hdcom

// Geometry/auxiliary.h of the reference
namespace aux {
using hdcom::zfill_int2string;
}  // namespace aux

namespace denoise {

class IterativeNLM_GPU {
public:
    int n_parallelslices = 0;
    bool resumed = false;
    int status = INLM_OK;

    IterativeNLM_GPU() = default;
    IterativeNLM_GPU(const IterativeNLM_GPU&) = delete;
    IterativeNLM_GPU& operator=(const IterativeNLM_GPU&) = delete;
    ~IterativeNLM_GPU() { free_device(); }

    // As the reference (iternlm_gpu.cu:1440-1566): params->gpu.n_gpus is
    // clipped to the devices from deviceID on; returns -1 without a CUDA
    // device, -2 on a CUDA error, else n_parallelslices: nz when the whole
    // stack is resident on one GPU (Run_GaussianNoise), fewer slices when the
    // stack is split over n_gpus > 1 devices (ceil(nz / n_gpus)) or does not
    // fit one device (the slab depth that fits); the caller then runs the
    // host-RAM Run_GaussianNoise_GPUBlocks per iteration.
    int configure_device(int shape[3], protocol::DenoiseParameters* params) {
        int ndev = 0;
        inlm_device_count(&ndev);
        if (ndev < 1) {
            params->gpu.n_gpus = 0;
            return -1;
        }
        params->gpu.n_gpus = std::max(1, std::min(ndev - params->gpu.deviceID, params->gpu.n_gpus));
        std::vector<int> ids;
        for (int i = 0; i < params->gpu.n_gpus; i++) ids.push_back(params->gpu.deviceID + i);
        return configure_devices(shape, params, ids);
    }
    // The same over an explicit device list (ids may repeat). slab_slices > 0
    // and below nz (one device): z-slabs of that depth even if the stack fits.
    int configure_devices(int shape[3], protocol::DenoiseParameters* params, const std::vector<int>& ids,
                          int slab_slices = 0) {
        free_device();
        if (ids.empty()) return -1;
        for (int i = 0; i < 3; i++) shape_[i] = shape[i];
        ids_ = ids;
        q_ = protocol::to_inlm(*params);
        q_.device_id = ids[0];
        if (ids.size() > 1) {
            // the reference's slab per GPU: ceil(nz / n_gpus) (iternlm_gpu.cu:1530-1532)
            return n_parallelslices = (shape[2] + (int)ids.size() - 1) / (int)ids.size();
        }
        if (slab_slices > 0 && slab_slices < shape[2]) return n_parallelslices = slab_slices;
        status = inlm_denoiser_create(shape, &q_, &h_);
        if (status == INLM_ERR_NODEVICE) return -1;
        if (status == INLM_ERR_NOMEM) {
            // z-slabs that fit: two sub-volumes (slab + halos) of raw, previous
            // iterate, result and staging, 16 bytes per voxel each
            status = INLM_OK;
            size_t free_b = 0, total_b = 0;
            if (inlm_device_memory(ids[0], &free_b, &total_b)) return -2;
            const long long plane = (long long)shape[0] * shape[1];
            const int pz = std::min(params->nslices / 2, params->radius_searchspace[2]) +
                           params->radius_patchspace[2];
            const int halo = (std::max(pz, 1) + 7) / 8 * 8;
            long long slab = (long long)(0.7 * (double)free_b / (32.0 * (double)plane)) - 2 * halo;
            slab = slab / 8 * 8;
            if (slab < 8) {
                protocol::report(INLM_ERR_NOMEM, "configure_device");
                return -2;
            }
            return n_parallelslices = (int)std::min<long long>(slab, shape[2] - 1);
        }
        if (protocol::report(status, "configure_device")) return -2;
        return n_parallelslices = shape[2];
    }
    void set_sigma(float* sigmalist, int /*shape*/[3]) {
        if (h_) {
            status = protocol::report(inlm_set_sigma(h_, sigmalist), "set_sigma");
        } else {
            sigma_.assign(sigmalist, sigmalist + shape_[2]);
            sigma_pending_ = true;
            status = INLM_OK;
        }
    }
    void Run_GaussianNoise(int iter, float* instack, int /*shape*/[3], protocol::DenoiseParameters*) {
        status = protocol::report(inlm_run_iteration(h_, iter, iter == 1 ? instack : nullptr),
                                  "Run_GaussianNoise");
    }
    // Host-RAM blocks (iternlm_gpu.cu:1729-1886): iteration iter of the whole
    // stack from instack and, after iteration 1, the previous iterate held in
    // `previous`; the result is left in `previous` (a malloc'd buffer of nz
    // slices, as the reference driver passes it). The result is the exact
    // iterate: unlike the reference, later blocks do not read slices that
    // earlier blocks of the same iteration have already overwritten. Under
    // --resume an iteration whose slices are all on disk in
    // params->io.active_outpath is read back instead (resumed = true).
    void Run_GaussianNoise_GPUBlocks(int iter, float* instack, float*& previous, int shape[3],
                                     protocol::DenoiseParameters* params) {
        resumed = false;
        const long long nstack = (long long)shape[0] * shape[1] * shape[2];
        if (params->io.resume &&
            hdcom::iteration_on_disk(params->io.active_outpath, params->io.firstslice, params->io.lastslice)) {
            float* r = hdcom::read_iteration(params->io.active_outpath, params->io.firstslice,
                                             params->io.lastslice, shape);
            if (!r) {
                status = INLM_ERR_IO;
                return;
            }
            free(previous);
            previous = r;
            resumed = true;
            std::cout << "iteration " << iter << " read in from disk" << std::endl;
            status = INLM_OK;
            return;
        }
        if (!b_) {
            status = protocol::report(inlm_blocks_create(shape_, &q_, (int)ids_.size(), ids_.data(),
                                                         n_parallelslices, &b_),
                                      "Run_GaussianNoise_GPUBlocks");
            if (status) return;
        }
        if (sigma_pending_) {
            status = protocol::report(inlm_blocks_set_sigma(b_, sigma_.data()), "set_sigma");
            if (status) return;
            sigma_pending_ = false;
        }
        if (iter == 1) {
            status = protocol::report(inlm_blocks_run_iteration(b_, 1, instack, nullptr, previous),
                                      "Run_GaussianNoise_GPUBlocks");
            return;
        }
        if (!spare_) spare_ = (float*)malloc(nstack * sizeof(float));
        if (!spare_) {
            status = protocol::report(INLM_ERR_NOMEM, "Run_GaussianNoise_GPUBlocks");
            return;
        }
        status = protocol::report(inlm_blocks_run_iteration(b_, iter, instack, previous, spare_),
                                  "Run_GaussianNoise_GPUBlocks");
        if (status == INLM_OK) std::swap(previous, spare_);  // both malloc'd; the old one is the next spare
    }
    // Disk blocks (iternlm_gpu.cu:1887-2115): slices re-read from files every
    // iteration. Not built: the host-RAM overload covers stacks larger than
    // device memory.
    void Run_GaussianNoise_GPUBlocks(int, std::vector<std::string>&, std::vector<std::string>&, int[3],
                                     protocol::DenoiseParameters*) {
        status = INLM_ERR_UNSUPPORTED;
        std::cout << "Error! disk-block mode (--blockwise_host) is not built; the stack is streamed "
                     "from host memory instead"
                  << std::endl;
    }
    // --resume: a finished iteration read back from disk (iternlm_gpu.cu:1665-1697)
    void set_result(int iter, const float* result, const float* instack) {
        status = protocol::report(inlm_set_result(h_, iter, result, instack), "set_result");
    }
    void get_result(float* output, int /*shape*/[3]) {
        status = protocol::report(inlm_get_result(h_, output), "get_result");
    }
    void free_device() {
        if (h_) inlm_denoiser_destroy(h_);
        h_ = nullptr;
        if (b_) inlm_blocks_destroy(b_);
        b_ = nullptr;
        free(spare_);
        spare_ = nullptr;
        sigma_pending_ = false;
    }

private:
    inlm_denoiser* h_ = nullptr;
    inlm_blocks* b_ = nullptr;
    inlm_params q_{};
    std::vector<int> ids_;
    int shape_[3] = {0, 0, 0};
    std::vector<float> sigma_;
    bool sigma_pending_ = false;
    float* spare_ = nullptr;
};

}  // namespace denoise

namespace noise {

class NoiseLevel {
public:
    int status = INLM_OK;

    NoiseLevel(uint64_t n_samples, int patchsize, int shape[3])
        : n_samples_(n_samples), patchsize_(patchsize) {
        for (int i = 0; i < 3; i++) shape_[i] = shape[i];
    }
    ~NoiseLevel() {
        if (h_) inlm_noise_destroy(h_);
    }
    NoiseLevel(const NoiseLevel&) = delete;
    NoiseLevel& operator=(const NoiseLevel&) = delete;

    // malloc'd float[nz] the caller frees; NULL on error. Writes the chosen
    // second value to params->noiselevel.sigma[1] in semimanual mode
    // (noiselevel.cpp:74).
    float* get_noiselevel(float* stack, std::vector<std::string>& /*filelist*/,
                          protocol::DenoiseParameters* params) {
        inlm_params q = protocol::to_inlm(*params);
        if (!h_) {
            status = protocol::report(inlm_noise_create(shape_, n_samples_, patchsize_, q.noise_seed,
                                                        q.device_id, &h_),
                                      "NoiseLevel");
            if (status) return nullptr;
        }
        float* sigma = (float*)malloc(sizeof(float) * shape_[2]);
        status = protocol::report(inlm_noise_estimate(h_, &q, stack, 0, sigma), "get_noiselevel");
        if (status) {
            free(sigma);
            return nullptr;
        }
        params->noiselevel.sigma[1] = q.sigma[1];
        return sigma;
    }

private:
    uint64_t n_samples_;
    int patchsize_;
    int shape_[3];
    inlm_noise* h_ = nullptr;
};

}  // namespace noise

namespace hdcom {

// The slice-sequence and noise-file members the driver calls.
class HdCommunication {
public:
    int status = INLM_OK;

    // {"missing"} / {"no tif"} on failure, as the reference signals it; the
    // list holds the input path (the library enumerates slices itself).
    std::vector<std::string> GetFilelist_And_ImageSequenceDimensions(const std::string& path,
                                                                      int outshape[3], bool& is_rgb) {
        struct stat st;
        if (stat(path.c_str(), &st) != 0) return {"missing"};
        int spp = 1;
        status = inlm_tiff_shape(path.c_str(), outshape, &spp);
        if (status != INLM_OK) {
            if (S_ISDIR(st.st_mode) && std::string(inlm_last_error()).find("No tif-file") != std::string::npos)
                return {"no tif"};
            protocol::report(status, "reading input");
            return {"missing"};
        }
        is_rgb = spp == 3 || spp == 4;
        return {path};
    }
    // Slices first..last (inclusive) of the stack; malloc'd, NULL on error.
    float* Get3DTifSequence_32bitPointer(const std::string& path, int outshape[3], int first, int last) {
        const size_t n = (size_t)outshape[0] * outshape[1] * (size_t)(last - first + 1);
        float* out = (float*)malloc(n * sizeof(float));
        status = protocol::report(inlm_tiff_read(path.c_str(), first, last, out, n), "reading stack");
        if (status) {
            free(out);
            return nullptr;
        }
        return out;
    }
    // The reference's overloads on its file list (one entry here: the input path).
    float* Get3DTifSequence_32bitPointer(std::vector<std::string>& filelist, int outshape[3], int first, int last) {
        return Get3DTifSequence_32bitPointer(filelist.empty() ? std::string() : filelist[0], outshape, first, last);
    }
    // A whole stack or ImageJ multi-page file (hdcommunication.cpp:1000-1060).
    float* GetTif_unknowndim_32bit(const std::string& path, int outshape[3], bool /*dspprogress*/ = false) {
        int spp = 1;
        status = protocol::report(inlm_tiff_shape(path.c_str(), outshape, &spp), "reading input");
        if (status) return nullptr;
        return Get3DTifSequence_32bitPointer(path, outshape, 0, outshape[2] - 1);
    }
    // The slices of an output directory, for the disk-block modes (the list
    // names the directory: the library enumerates its slices itself).
    std::vector<std::string> GetFilelist(const std::string& path, int /*outshape*/[3]) { return {path}; }
    void SaveTifSequence_32bit(int z0, float* image, int imgshape[3], const std::string& path,
                               const std::string& name, bool /*dspprogress*/) {
        status = protocol::report(
            inlm_tiff_write_sequence(image, imgshape, z0, path.c_str(), name.c_str(), 0), "saving stack");
    }
    void SaveTifSequence_as16bit(int z0, float* image, int imgshape[3], const std::string& path,
                                 const std::string& name, bool /*dspprogress*/) {
        status = protocol::report(
            inlm_tiff_write_sequence(image, imgshape, z0, path.c_str(), name.c_str(), 1), "saving stack");
    }
    // "n,value" lines (hdcommunication.cpp:1736-1746)
    void SaveNoisefile(const float* y, int length, const std::string& path, const std::string& name) {
        std::string cmd_dir = path;
        mkdirs(cmd_dir);
        std::ofstream out(path + "/" + name + ".csv");
        for (int64_t n = 0; n < length; n++) out << n << "," << y[n] << "\n";
    }
    // true when the file holds exactly nz values (hdcommunication.cpp:1747-1786)
    bool ReadNoisefile(float*& sigma, int shape[3], const std::string& file) {
        std::ifstream in(file);
        if (!in.is_open()) return false;
        std::vector<double> ys;
        std::string line;
        while (std::getline(in, line)) {
            std::stringstream ss(line);
            std::string a, b;
            std::getline(ss, a, ',');
            std::getline(ss, b, ',');
            ys.push_back(atof(b.c_str()));
        }
        if ((int)ys.size() != shape[2]) return false;
        sigma = (float*)malloc(sizeof(float) * shape[2]);
        for (int i = 0; i < shape[2]; i++) sigma[i] = (float)ys[i];
        return true;
    }
    static void mkdirs(const std::string& path) {
        std::string cur;
        for (size_t i = 0; i < path.size(); i++) {
            cur += path[i];
            if (path[i] == '/' && cur.size() > 1) mkdir(cur.c_str(), 0777);
        }
        mkdir(path.c_str(), 0777);
    }
};

}  // namespace hdcom

namespace denoise {

// The reference's CPU filter class (Denoiser/iternlm_cpu.h:30-157), which its
// driver falls back to without a CUDA device. This library filters on the GPU
// only: the members report an error and return the caller's buffer.
class IterativeNLM_CPU {
public:
    int status = INLM_OK;
    void print_estimatedmemory(int /*shape*/[3], protocol::DenoiseParameters*) {}
    float* Run_GaussianNoise(int, float*&, float*& previous, float*, int[3], protocol::DenoiseParameters*) {
        return unsupported(previous);
    }
    float* Run_GaussianNoise_unrolled(int, float*&, float*& previous, float*, int[3], protocol::DenoiseParameters*) {
        return unsupported(previous);
    }
    void Run_GaussianNoise_blocks(int, std::vector<std::string>&, std::vector<std::string>&, float*, int[3],
                                  protocol::DenoiseParameters*) {
        unsupported(nullptr);
    }
    void Run_GaussianNoise_blocks_unrolled(int, std::vector<std::string>&, std::vector<std::string>&, float*, int[3],
                                           protocol::DenoiseParameters*) {
        unsupported(nullptr);
    }

private:
    float* unsupported(float* p) {
        status = INLM_ERR_UNSUPPORTED;
        std::cout << "Error! This library has no CPU filter (it runs on CUDA devices only)" << std::endl;
        return p;
    }
};

}  // namespace denoise

namespace color_denoise {

struct ColorSave {
    std::string dir, name;
    int nx, ny;
    int status;
};

// saves one iteration of the colour job (color_denoising.h:73-84)
inline void save_color_iteration(int iter, const float* r, const float* g, const float* b, void* user) {
    ColorSave* s = static_cast<ColorSave*>(user);
    const int rc = inlm_tiff_write_rgb(s->dir.c_str(), (s->name + "_iter" + hdcom::zfill_int2string(iter, 2)).c_str(),
                                       r, g, b, s->nx, s->ny);
    if (rc != INLM_OK) s->status = protocol::report(rc, "saving iteration");
}

// The colour driver (Color/color_denoising.h:19-150): every RGB image of the
// input (filelist[0]: one .tif file or a directory of them), 2D, on the GPU.
// Returns 0, or a negative value on error.
inline int run_colorimage_denoising(std::vector<std::string>& filelist, std::string outpath,
                                    protocol::DenoiseParameters* params) {
    const std::string inpath = filelist.empty() ? std::string() : filelist[0];
    std::vector<std::string> files;
    const bool single = inpath.size() >= 3 && (inpath.substr(inpath.size() - 3) == "tif" ||
                                               (inpath.size() >= 4 && inpath.substr(inpath.size() - 4) == "tiff"));
    if (single) {
        files.push_back(inpath);
    } else {
        std::error_code ec;
        for (const auto& e : std::filesystem::directory_iterator(inpath, ec)) {
            const std::string f = e.path().string();
            if ((f.size() > 4 && f.substr(f.size() - 4) == ".tif") || (f.size() > 5 && f.substr(f.size() - 5) == ".tiff"))
                files.push_back(f);
        }
        std::sort(files.begin(), files.end());
    }
    // the colour driver's fixed settings (color_denoising.h:25-28)
    params->radius_patchspace[2] = 0;
    params->radius_searchspace[2] = 0;
    params->nslices = 1;
    params->noiselevel.n_samples = 2048;
    const inlm_params q = protocol::to_inlm(*params);
    const inlm_color_params cp = {params->color.stabilize_variance ? 1 : 0, params->color.independent_channels ? 1 : 0,
                                  params->color.average_channelsigma ? 1 : 0};
    for (const std::string& file : files) {
        std::cout << "--------------------------------------" << std::endl;
        const size_t slash = file.rfind('/');
        std::string name = file.substr(slash == std::string::npos ? 0 : slash + 1);
        name = name.substr(0, name.rfind('.'));
        std::cout << "image: " << name << std::endl;
        int shape[2];
        if (protocol::report(inlm_tiff_read_rgb(file.c_str(), shape, nullptr, nullptr, nullptr, 0), "reading image"))
            return -1;
        const size_t n = (size_t)shape[0] * shape[1];
        std::vector<float> in(3 * n), out(3 * n);
        if (protocol::report(inlm_tiff_read_rgb(file.c_str(), shape, in.data(), in.data() + n, in.data() + 2 * n, n),
                             "reading image"))
            return -1;
        ColorSave save{outpath + "/denoise_iterations/", name, shape[0], shape[1], INLM_OK};
        float s_first[3], s_last[3];
        const int rc = inlm_rgb_denoise(shape[0], shape[1], &q, &cp, in.data(), in.data() + n, in.data() + 2 * n,
                                        out.data(), out.data() + n, out.data() + 2 * n,
                                        params->io.cleanup ? nullptr : save_color_iteration, &save, s_first, s_last);
        if (protocol::report(rc, "rgb_denoise") || save.status) return -2;
        std::cout << "initial noise level: " << s_first[0] << ", " << s_first[1] << ", " << s_first[2] << std::endl;
        std::cout << "final noise level: " << s_last[0] << ", " << s_last[1] << ", " << s_last[2] << std::endl;
        if (protocol::report(inlm_tiff_write_rgb(outpath.c_str(), (name + "_denoised").c_str(), out.data(),
                                                 out.data() + n, out.data() + 2 * n, shape[0], shape[1]),
                             "saving image"))
            return -1;
    }
    std::cout << "--------------------------------------" << std::endl;
    return 0;
}

}  // namespace color_denoise

