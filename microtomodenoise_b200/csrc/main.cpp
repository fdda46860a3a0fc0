// iterNLM command line on the B200 library: the flags, flow, output layout
// and log of the reference driver (iterNLM_v0.3/main.cpp:31-599), with the
// filter and noise estimates on the GPU through iternlm.hpp.
//
//   iterNLM -i <slice dir | stack.tif> [-o <outdir>] [flags]
//
// Output: <outdir>/denoise-iterationNN/denoised####.tif per iteration (only
// the last one, written to <outdir> itself, with --cleanup),
// <outdir>/noise_vs_sliceNN.csv, and a run record appended to logfile.txt one
// level above <outdir>; with --color, <outdir>/<image>_denoised.tif per RGB
// image (and <outdir>/denoise_iterations/<image>_iterNN.tif without
// --cleanup). Not built: the CPU filter (-gpus 0).
// Additions: -precision f32|f16, -seed N (noise sample draw), -slab N
// (stream the stack through one device in z-slabs of N slices; without it
// slabs are used only when the stack does not fit), -gpulist a,b,... (the
// devices of the multi-GPU split; -gpus N takes N devices from -gpu0).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "iternlm.hpp"

using std::cout;
using std::endl;
using std::string;

int main(int argc, char* argv[]) {
    string inpath = "", outpath = "";
    bool verbose = false;
    int slab_depth = 0;  // -slab N: stream z-slabs of N slices even when the stack fits
    std::vector<int> gpulist;
    protocol::DenoiseParameters params;
    string rootpath;

    for (int i = 1; i < argc; i++) {
        const string a = argv[i];
        auto next = [&]() -> const char* {
            if (i + 1 >= argc) {
                cout << "Error! " << a << " needs a value" << endl;
                exit(-1);
            }
            return argv[++i];
        };
        if (a == "-i" || a == "-input") inpath = next();
        else if (a == "-o" || a == "-output") outpath = next();
        else if (a == "-r" || a == "-resume") {
            const string v = next();
            if (v == "false" || v == "False") params.io.resume = false;
            else if (v == "true" || v == "True") params.io.resume = true;
        } else if (a == "--resume") params.io.resume = true;
        else if (a == "-fs" || a == "-firstslice") params.io.firstslice = atoi(next());
        else if (a == "-ls" || a == "-lastslice") params.io.lastslice = atoi(next());
        else if (a == "--16bit") params.io.save_type = "16bit";
        else if (a == "--cleanup") params.io.cleanup = true;
        else if (a == "--color" || a == "--rgb") params.io.rgb = true;
        else if (a == "-aniso" || a == "-anisotropy") params.z_anisotropy = (float)atof(next());
        else if (a == "-maxiter" || a == "-iter" || a == "-iterations") params.maxiterations = atoi(next());
        else if (a == "-slices" || a == "-nslices") params.nslices = atoi(next());
        else if (a == "-a" || a == "-alpha") params.alpha = (float)atof(next());
        else if (a == "-search") {
            const int r = atoi(next());
            params.radius_searchspace[0] = params.radius_searchspace[1] = params.radius_searchspace[2] = r;
        } else if (a == "-search0") params.radius_searchspace[0] = atoi(next());
        else if (a == "-search1") params.radius_searchspace[1] = atoi(next());
        else if (a == "-search2") params.radius_searchspace[2] = atoi(next());
        else if (a == "-patch") {
            const int r = atoi(next());
            params.radius_patchspace[0] = params.radius_patchspace[1] = params.radius_patchspace[2] = r;
        } else if (a == "-patch0") params.radius_patchspace[0] = atoi(next());
        else if (a == "-patch1") params.radius_patchspace[1] = atoi(next());
        else if (a == "-patch2") params.radius_patchspace[2] = atoi(next());
        else if (a == "--independent") params.color.independent_channels = true;
        else if (a == "-cpus" || a == "-n_cpus") params.cpu.max_threads = atoi(next());
        else if (a == "-gpus" || a == "-n_gpus" || a == "-ngpus") params.gpu.n_gpus = atoi(next());
        else if (a == "-gpu0") params.gpu.deviceID = atoi(next());
        else if (a == "-threads") params.gpu.threadsPerBlock = atoi(next());
        else if (a == "--noblocks") params.cpu.blockwise = params.gpu.blockwise_host = false;
        else if (a == "--blocks") params.cpu.blockwise = params.gpu.blockwise_host = true;
        else if (a == "--unroll") params.cpu.unrolled_patchspace = true;
        else if (a == "--verbose" || a == "--v") verbose = true;
        else if (a == "-noise" || a == "-noisemode") params.noiselevel.mode = next();
        else if (a == "-sigma" || a == "-s") {
            params.noiselevel.sigma[0] = (float)atof(next());
            params.noiselevel.sigma[1] = params.noiselevel.sigma[0];
        } else if (a == "-sigma0" || a == "-s0") params.noiselevel.sigma[0] = (float)atof(next());
        else if (a == "-sigma1" || a == "-s1") params.noiselevel.sigma[1] = (float)atof(next());
        else if (a == "-nsamples" || a == "-noise_samples") params.noiselevel.n_samples = (uint64_t)atoi(next());
        else if (a == "-noisepatch") params.noiselevel.patchsize = atoi(next());
        else if (a == "-noiseshift") params.noiselevel.stds_from_mean = (float)atof(next());
        else if (a == "-mask" || a == "-mask_diameter") params.noiselevel.circular_mask_diameter = atoi(next());
        else if (a == "--continuous") params.noiselevel.continuous_estimate = true;
        else if (a == "--preserve_detail") {
            params.noiselevel.continuous_estimate = true;
            params.alpha = 0.0f;
            params.noiselevel.stds_from_mean = 4.f;
            params.maxiterations = 6;
        } else if (a == "--nopoisson") params.color.stabilize_variance = false;
        else if (a == "--noaverage") params.color.average_channelsigma = false;
        else if (a == "-precision") params.gpu.precision = next();
        else if (a == "-seed") params.noiselevel.seed = (unsigned int)strtoul(next(), nullptr, 10);
        else if (a == "-slab") slab_depth = atoi(next());
        else if (a == "-gpulist") {
            // explicit devices of the multi-GPU split, e.g. 0,1,2,3 (may repeat)
            gpulist.clear();
            const string v = next();
            size_t pos = 0;
            while (pos <= v.size()) {
                const size_t c = v.find(',', pos);
                gpulist.push_back(atoi(v.substr(pos, c == string::npos ? string::npos : c - pos).c_str()));
                if (c == string::npos) break;
                pos = c + 1;
            }
        }
        else if (a == "-h" || a == "-help" || a == "--help") {
            cout << "iterNLM (B200): iterative 3D nonlocal means for tomographic stacks.\n"
                    "usage: iterNLM -i <slice directory | stack.tif> [-o <outdir>] [-iter N] "
                    "[-patch R] [-search R] [-nslices N] [-alpha A] [-noise z-adaptive|global|manual|semimanual] "
                    "[-sigma S] [-fs N -ls N] [--16bit] [--cleanup] [--resume] [-precision f32|f16] "
                    "[-seed N]"
                 << endl;
            return 0;
        } else if (inpath.empty()) inpath = a;
    }
    if (inpath.empty()) {
        cout << "Error! No input given: iterNLM -i <slice directory | stack.tif>" << endl;
        return -1;
    }
    rootpath = inpath.substr(0, inpath.rfind('/', inpath.length() - 2) + 1);
    if (outpath.empty()) outpath = rootpath + "/denoised/";
    else rootpath = outpath.substr(0, outpath.rfind('/', outpath.length() - 2) + 1);

    const auto time0 = std::chrono::high_resolution_clock::now();

    int shape[3];
    hdcom::HdCommunication hdcom;
    bool is_rgb = false;
    std::vector<string> filelist = hdcom.GetFilelist_And_ImageSequenceDimensions(inpath, shape, is_rgb);
    if (filelist[0] == "missing") {
        cout << "Error! Directory or file not found! Please provide a valid input with the -i argument" << endl;
        return -1;
    }
    if (filelist[0] == "no tif") {
        cout << "Error! No tif-file in directory! Please provide a valid input with the -i argument" << endl;
        return -1;
    }
    if (params.io.rgb) {
        cout << "Switching to RGB-Denoiser!" << endl;
        std::vector<string> files{inpath};
        return color_denoise::run_colorimage_denoising(files, outpath, &params);
    }
    if (is_rgb) {
        cout << "Error! RGB input: run with --color" << endl;
        return -1;
    }
    if (params.gpu.n_gpus <= 0) {
        cout << "Error! This program filters on the GPU only (-gpus 0 asks for the CPU filter)" << endl;
        return -1;
    }
    if (gpulist.size() == 1) params.gpu.deviceID = gpulist[0];
    if (shape[2] == 1) {
        params.radius_patchspace[2] = 0;
        params.radius_searchspace[2] = 0;
    }

    cout << "--------------------------------------------------" << endl;
    cout << "iterNLM (B200) for " << inpath << endl;
    cout << "--------------------------------------------------" << endl;
    cout << "alpha: " << params.alpha << endl;
    cout << "search_radius: " << params.radius_searchspace[0] << " " << params.radius_searchspace[1] << " "
         << params.radius_searchspace[2] << endl;
    cout << "n_slices: " << params.nslices << endl;
    cout << "patch_radius: " << params.radius_patchspace[0] << " " << params.radius_patchspace[1] << " "
         << params.radius_patchspace[2] << endl;
    cout << "noise estimate: " << params.noiselevel.mode << endl;
    cout << "image shape: " << shape[0] << "x" << shape[1] << "x" << shape[2] << endl;
    if (params.z_anisotropy != 1.f) cout << "vxl anisotropy: " << params.z_anisotropy << endl;
    if (params.gpu.precision != "f32") cout << "precision: " << params.gpu.precision << endl;
    cout << "--------------------------------------------------" << endl;

    // slice range (main.cpp:276-298); -1 at one end means that end of the stack
    if (params.io.firstslice != -1 || params.io.lastslice != -1) {
        params.io.firstslice = std::max(0, params.io.firstslice);
        params.io.lastslice = params.io.lastslice == -1 ? shape[2] - 1 : std::min(shape[2] - 1, params.io.lastslice);
        if (params.io.lastslice < params.io.firstslice) {
            cout << "Error! Empty slice range" << endl;
            return -1;
        }
    } else {
        params.io.firstslice = 0;
        params.io.lastslice = shape[2] - 1;
    }
    float* instack = hdcom.Get3DTifSequence_32bitPointer(inpath, shape, params.io.firstslice, params.io.lastslice);
    if (!instack) return -1;
    shape[2] = params.io.lastslice - params.io.firstslice + 1;
    const long long nstack = (long long)shape[0] * shape[1] * shape[2];
    const bool save16 = params.io.save_type == "16bit";
    auto save = [&](float* img, const string& dir) {
        if (save16) hdcom.SaveTifSequence_as16bit(params.io.firstslice, img, shape, dir, "denoised", false);
        else hdcom.SaveTifSequence_32bit(params.io.firstslice, img, shape, dir, "denoised", false);
        return hdcom.status;
    };
    auto iterdir = [&](int iter) {
        if (iter == params.maxiterations && params.io.cleanup) return outpath;
        return outpath + "/denoise-iteration" + hdcom::zfill_int2string(iter, 2) + "/";
    };

    // devices: -gpulist, else -gpus N from -gpu0 (the reference's n_gpus
    // mode, default 2), clipped to the devices present
    int n_devices = 0;
    if (inlm_device_count(&n_devices) != INLM_OK) n_devices = 0;
    std::vector<int> ids = gpulist;
    if (ids.empty())
        for (int i = 0; i < std::min(params.gpu.n_gpus, n_devices - params.gpu.deviceID); i++)
            ids.push_back(params.gpu.deviceID + i);
    if (ids.empty() && n_devices > 0) ids.push_back(params.gpu.deviceID % n_devices);
    // a split needs every part at least one z halo deep (8-slice units split
    // evenly; the last part may lose up to 7 slices to the stack's end)
    const int zpad = std::min(params.nslices / 2, params.radius_searchspace[2]) + params.radius_patchspace[2];
    const int halo = (std::max(zpad, 1) + 7) / 8 * 8;
    const int units = (shape[2] + 7) / 8;
    if (ids.size() > 1 && !(8 * (units / (int)ids.size()) - 7 >= halo && shape[2] >= 16 * (int)ids.size()))
        ids.resize(1);

    denoise::IterativeNLM_GPU gpu;
    int n_parallelslices = n_devices > 0 ? gpu.configure_devices(shape, &params, ids) : -1;
    if (n_parallelslices == -2) return -2;
    if (n_parallelslices == -1) {
        cout << "Error! No CUDA device found (this program has no CPU filter)" << endl;
        return -1;
    }
    // -slab N below the stack depth: z-slab streaming on one device
    if (ids.size() == 1 && slab_depth > 0 && slab_depth < shape[2]) {
        gpu.free_device();
        n_parallelslices = gpu.configure_devices(shape, &params, ids, slab_depth);
        if (n_parallelslices < 0) return -2;
    }
    const bool blocks = n_parallelslices < shape[2];
    if (blocks) {
        if (ids.size() > 1) cout << "Processing " << shape[2] << " slices on " << ids.size() << " GPUs" << endl;
        else cout << "Streaming z-slabs of " << n_parallelslices << " slices through the GPU" << endl;
    }

    float *sigma0 = nullptr, *sigma1 = nullptr;
    float* output = (float*)malloc(nstack * sizeof(float));
    {
        noise::NoiseLevel noise(params.noiselevel.n_samples, params.noiselevel.patchsize, shape);
        auto estimate = [&](float* stack, float*& sigma, int index, const char* what) {
            bool available = false;
            if (params.io.resume)
                available = hdcom.ReadNoisefile(sigma, shape, outpath + "/noise_vs_slice" +
                                                                  hdcom::zfill_int2string(index, 2) + ".csv");
            if (!available) {
                cout << what << "...\r";
                cout.flush();
                sigma = noise.get_noiselevel(stack, filelist, &params);
                if (!sigma) return false;
                if (!params.io.cleanup || verbose)
                    hdcom.SaveNoisefile(sigma, shape[2], outpath, "noise_vs_slice" + hdcom::zfill_int2string(index, 2));
            } else {
                cout << "Read in noise level " << index << " from file!" << endl;
            }
            return true;
        };
        auto run = [&](int iter) {
            params.io.active_outpath = iterdir(iter);
            const auto t0 = std::chrono::high_resolution_clock::now();
            if (blocks) {
                // host-RAM blocks (main.cpp:377-384, 471-478): the result lands
                // in output; --resume reads a finished iteration back
                gpu.Run_GaussianNoise_GPUBlocks(iter, instack, output, shape, &params);
                if (gpu.status) return false;
                if (gpu.resumed) return true;
            } else {
                if (params.io.resume &&
                    hdcom::iteration_on_disk(params.io.active_outpath, params.io.firstslice, params.io.lastslice)) {
                    float* r = hdcom::read_iteration(params.io.active_outpath, params.io.firstslice,
                                                     params.io.lastslice, shape);
                    if (!r) return false;
                    gpu.set_result(iter, r, instack);
                    std::memcpy(output, r, nstack * sizeof(float));
                    free(r);
                    cout << "iteration " << iter << " read in from disk" << endl;
                    return gpu.status == INLM_OK;
                }
                gpu.Run_GaussianNoise(iter, instack, shape, &params);
                if (gpu.status) return false;
                gpu.get_result(output, shape);
                if (gpu.status) return false;
            }
            const std::chrono::duration<double> dt = std::chrono::high_resolution_clock::now() - t0;
            cout << "iteration " << iter << " took " << dt.count() << " s                          " << endl;
            if (iter == 1 || !params.io.cleanup || iter == params.maxiterations)
                if (save(output, params.io.active_outpath)) return false;
            return true;
        };

        if (!estimate(instack, sigma0, 0, "estimating initial noise level")) return -2;
        gpu.set_sigma(sigma0, shape);
        if (gpu.status) return -2;
        cout << "initial noise level (slice " << shape[2] / 2 << "): " << sigma0[shape[2] / 2] << "          " << endl;

        if (!run(1)) return -2;
        if (params.maxiterations > 1) {
            if (!estimate(output, sigma1, 1, "reestimating noise level")) return -2;
            cout << "2nd noise level (slice " << shape[2] / 2 << "): " << sigma1[shape[2] / 2] << "          " << endl;
            for (int i = 0; i < shape[2]; i++) sigma1[i] = params.alpha * sigma0[i] + (1.f - params.alpha) * sigma1[i];
            gpu.set_sigma(sigma1, shape);
            if (gpu.status) return -2;
        }
        for (int iter = 2; iter <= params.maxiterations; iter++) {
            if (!run(iter)) return -2;
            if (params.noiselevel.continuous_estimate && params.maxiterations > iter + 1) {
                free(sigma1);
                sigma1 = nullptr;
                if (!estimate(output, sigma1, iter, "reestimating noise level")) return -2;
                cout << "noise level " << iter << " (slice " << shape[2] / 2 << "): " << sigma1[shape[2] / 2]
                     << "          " << endl;
                for (int i = 0; i < shape[2]; i++) sigma1[i] = params.alpha * sigma0[i] + (1.f - params.alpha) * sigma1[i];
                gpu.set_sigma(sigma1, shape);
                if (gpu.status) return -2;
            }
        }
    }

    // intermediate iterations are dropped with --cleanup (main.cpp:518-530)
    if (params.io.cleanup) {
        for (int iter = 1; iter < params.maxiterations; iter++) {
            std::error_code ec;
            std::filesystem::remove_all(outpath + "/denoise-iteration" + hdcom::zfill_int2string(iter, 2), ec);
        }
    }
    gpu.free_device();

    {
        const time_t now = time(nullptr);
        std::ofstream log(rootpath + "/logfile.txt", std::ios::app);
        log << ctime(&now);
        log << "ran iterNLM (B200) for " << inpath << "\n";
        log << "-------------------------------------------------------------------------\n";
        const int zc = shape[2] / 2;
        if (params.noiselevel.mode == "z-adaptive") {
            log << "    noise estimate: z-adaptive (moving window " << params.noiselevel.zwindow << ")\n";
            log << "    sigma0(slice " << zc << "): " << sigma0[zc] << "\n";
            if (params.maxiterations > 1 && sigma1) log << "    sigma1(slice " << zc << "): " << sigma1[zc] << "\n";
        } else {
            log << "    noise estimate: " << params.noiselevel.mode << "\n";
            log << "    sigma0: " << sigma0[zc] << "\n";
            if (params.maxiterations > 1 && sigma1) log << "    sigma1: " << sigma1[zc] << "\n";
        }
        log << "    alpha:  " << params.alpha << "\n";
        log << "    iterations: " << params.maxiterations << "\n";
        log << "    slices: " << params.nslices << "\n";
        log << "    patch space:  (" << params.radius_patchspace[0] << "," << params.radius_patchspace[1] << ","
            << params.radius_patchspace[2] << ")\n";
        log << "    search space: (" << params.radius_searchspace[0] << "," << params.radius_searchspace[1] << ","
            << params.radius_searchspace[2] << ")\n";
        log << "    precision: " << params.gpu.precision << "\n";
        log << "-------------------------------------------------------------------------\n\n";
    }
    free(instack);
    free(output);
    free(sigma0);
    free(sigma1);
    cout << "--------------------------------------------------" << endl;
    const std::chrono::duration<double> total = std::chrono::high_resolution_clock::now() - time0;
    cout << "execution took " << total.count() << " s" << endl;
    cout << "--------------------------------------------------" << endl;
    return 0;
}
