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

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
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

namespace denoise {

class IterativeNLM_GPU {
public:
    int n_parallelslices = 0;
    bool resumed = false;
    int status = INLM_OK;

    ~IterativeNLM_GPU() { free_device(); }

    // n_parallelslices (= nz: the whole stack is resident), -1 without a CUDA
    // device, -2 on a CUDA error, 0 when the stack does not fit in device
    // memory (the caller then streams it in z-slabs).
    int configure_device(int shape[3], protocol::DenoiseParameters* params) {
        free_device();
        const inlm_params q = protocol::to_inlm(*params);
        status = inlm_denoiser_create(shape, &q, &h_);
        if (status == INLM_ERR_NODEVICE) return -1;
        if (status == INLM_ERR_NOMEM) return n_parallelslices = 0;
        if (protocol::report(status, "configure_device")) return -2;
        return n_parallelslices = shape[2];
    }
    void set_sigma(float* sigmalist, int /*shape*/[3]) {
        status = protocol::report(inlm_set_sigma(h_, sigmalist), "set_sigma");
    }
    void Run_GaussianNoise(int iter, float* instack, int /*shape*/[3], protocol::DenoiseParameters*) {
        status = protocol::report(inlm_run_iteration(h_, iter, iter == 1 ? instack : nullptr),
                                  "Run_GaussianNoise");
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
    }

private:
    inlm_denoiser* h_ = nullptr;
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

inline std::string zfill_int2string(int v, unsigned int width) {
    std::string s = std::to_string(v);
    while (s.size() < width) s = "0" + s;
    return s;
}

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
