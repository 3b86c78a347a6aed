// gisspa_main: drop-in replacement of the reference's `./main <config>`
// (main.cu:1025-1299).  Same config keys, input list, Euler file, MRC inputs
// and byte-compatible output lines; the search itself runs through the C ABI
// (include/gisspa.h) on one GPU.
//
// Differences from the reference, all on failure paths: unreadable inputs
// are reported and the run stops with a non-zero exit code instead of being
// replaced by a 10x10 zero image (emdata_.cpp:185-203), and every micrograph
// is searched at its own size instead of the first micrograph's
// (main.cu:1108-1109, 1160).
#include <sys/stat.h>
#include <sys/types.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gisspa.h"
#include "refio.hpp"

using namespace gsdrv;

static void print_help() {
    printf("gisspa_main: GisSPA 2D template-matching search (B200).\n");
    printf("Usage: gisspa_main config_file\n");
    printf("All parameters are set in the config file, one \"key = value\" per line.\n");
    printf("Requested parameters:\n");
    printf("input            = input micrograph list (.lst) with ctf information\n");
    printf("template         = 2D projection templates (MRC stack)\n");
    printf("eulerfile        = euler file, \"alt az\" per template\n");
    printf("angpix           = pixel size in angstroms\n");
    printf("phistep          = in-plane rotation sampling, degrees\n");
    printf("kk               = overlapping density parameter, default is 3\n");
    printf("energy           = accelerating voltage in kV\n");
    printf("cs               = spherical aberration in mm\n");
    printf("Highres          = high resolution cut\n");
    printf("Lowres           = low resolution cut\n");
    printf("diameter         = target diameter in pixels\n");
    printf("Optional parameters:\n");
    printf("norm_type        = 0: score = peak / sigma per map; 1: per-pixel z-score over all templates and angles\n");
    printf("invert           = 0 / 1, invert contrast\n");
    printf("threshold        = score threshold, only scores >= it are written\n");
    printf("output           = output list file name\n");
    printf("first            = first micrograph index to process\n");
    printf("last             = one past the last micrograph index\n");
    printf("window_size      = window size cut from the micrograph\n");
    printf("GPU_ID           = CUDA device id\n");
    printf("phase_flip       = 1 to phase-flip and whiten the micrograph\n");
    printf("overlap          = overlap between windows, px\n");
}

// Create the directories on the way to `path` (main.cu:1007-1023).
static void create_outpath(const std::string& path) {
    for (size_t pos = 0; pos < path.size(); ++pos) {
        if (path[pos] != '/' || pos == 0) continue;
        mkdir(path.substr(0, pos).c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    }
}

static int fail(const char* what, gs_ctx* ctx, int st) {
    fprintf(stderr, "gisspa_main: %s failed: %s%s%s\n", what, gs_status_string(st), ctx ? ": " : "",
            ctx ? gs_ctx_last_error(ctx) : "");
    return 2;
}

int main(int argc, char** argv) {
    if (argc == 1 || (argv[1][0] == '-' && argv[1][1] == 'h')) {
        print_help();
        return 0;
    }
    Config cfg;
    if (!read_config(argv[1], &cfg)) {
        fprintf(stderr, "Error => Open config file failed : %s\n", argv[1]);
        return 1;
    }
    for (const auto& u : cfg.unknown) printf("Undefined option: %s .Abort.\n", u.c_str());
    const auto missing = missing_required(cfg);
    for (const auto& m : missing) printf("Error : %s is requested.\n", m.c_str());
    print_config(cfg);
    if (!missing.empty()) return 1;

    Euler eul;
    if (!read_euler(cfg.eulerf, &eul)) {
        fprintf(stderr, "Error => Open euler file failed : %s\n", cfg.eulerf.c_str());
        return 1;
    }
    const int ntmpl = (int)eul.alt.size();
    if (ntmpl == 0) {
        fprintf(stderr, "Error => no templates listed in %s\n", cfg.eulerf.c_str());
        return 1;
    }
    create_outpath(cfg.outlst);
    FILE* fp = fopen(cfg.outlst.c_str(), "wb");
    if (!fp) {
        printf("Out file create failed! %s\n", cfg.outlst.c_str());
        printf("Please confirm the path exists!\n");
        return 1;
    }

    // first micrograph: its CTF weights every template (main.cu:1106, 1129)
    CtfState ctf;
    LstEntry ent;
    int rc = read_lst_entry(cfg.inlst, cfg.first, &ent, &ctf);
    if (rc < 0) {
        fprintf(stderr, "Error %d occured reading entry %d of %s\n", rc, cfg.first, cfg.inlst.c_str());
        fclose(fp);
        return 1;
    }
    const CtfState ctf_first = ctf;

    // template stack: section (MRC) or image (EMAN HDF5) J for template J
    // (main.cu:182-223)
    Image t0;
    std::string err = read_image(cfg.temp2d, 0, &t0);
    if (!err.empty()) {
        fprintf(stderr, "%s\n", err.c_str());
        fclose(fp);
        return 1;
    }
    const int tx = t0.nx, ty = t0.ny;
    std::vector<float> stack((size_t)ntmpl * tx * ty);
    if (is_hdf5(cfg.temp2d)) {
        for (int J = 0; J < ntmpl; ++J) {
            Image tj;
            err = read_image(cfg.temp2d, J, &tj);
            if (!err.empty() || tj.nx != tx || tj.ny != ty || tj.nz != 1) {
                fprintf(stderr, "%s\n", err.empty() ? "template images differ in size" : err.c_str());
                fclose(fp);
                return 1;
            }
            memcpy(stack.data() + (size_t)J * tx * ty, tj.data.data(), sizeof(float) * tx * ty);
        }
    } else {
        Image all;
        err = read_mrc(cfg.temp2d, -1, &all);
        if (!err.empty() || all.nx != tx || all.ny != ty) {
            fprintf(stderr, "%s\n", err.empty() ? "template stack geometry mismatch" : err.c_str());
            fclose(fp);
            return 1;
        }
        for (int J = 0; J < ntmpl; ++J) {
            const int src = J < all.nz ? J : 0;  // an out-of-range section reads the stack from its start
            memcpy(stack.data() + (size_t)J * tx * ty, all.data.data() + (size_t)src * tx * ty,
                   sizeof(float) * tx * ty);
        }
    }

    gs_ctx* ctx = nullptr;
    int st = gs_ctx_create(cfg.device_id, &ctx);
    if (st != GS_OK) return fail("gs_ctx_create", nullptr, st);
    gs_params p;
    gs_params_default(&p);
    p.apix = cfg.apix; p.phi_step = cfg.phi_step; p.kk = cfg.kk; p.energy = cfg.energy; p.cs = cfg.cs;
    p.highres = cfg.highres; p.lowres = cfg.lowres; p.d_m = cfg.d_m; p.thres = cfg.thres;
    p.window_size = cfg.padding_size; p.overlap = cfg.overlap; p.phase_flip = cfg.phase_flip;
    p.norm_type = cfg.norm_type; p.invert = cfg.invert;
    const gs_ctf c0{ctf_first.defocus, ctf_first.dfdiff, ctf_first.dfang};
    st = gs_set_templates(ctx, &p, stack.data(), ntmpl, tx, ty, &c0);
    if (st != GS_OK) {
        fclose(fp);
        return fail("template preprocessing", ctx, st);
    }

    const auto t_start = std::chrono::steady_clock::now();
    for (int n = cfg.first; n < cfg.last; ++n) {
        rc = read_lst_entry(cfg.inlst, n, &ent, &ctf);
        if (rc < 0) {
            fprintf(stderr, "Error %d occured reading entry %d of %s\n", rc, n, cfg.inlst.c_str());
            fclose(fp);
            gs_ctx_destroy(ctx);
            return 1;
        }
        Image mic;
        err = read_image(ent.path, ent.nn, &mic);
        if (!err.empty()) {
            fprintf(stderr, "%s\n", err.c_str());
            fclose(fp);
            gs_ctx_destroy(ctx);
            return 1;
        }
        const gs_ctf cm{ctf.defocus, ctf.dfdiff, ctf.dfang};
        gs_pick* picks = nullptr;
        size_t np = 0;
        st = gs_search(ctx, mic.data.data(), mic.nx, mic.ny, &cm, &picks, &np);
        if (st != GS_OK) {
            fclose(fp);
            return fail("search", ctx, st);
        }
        // writeScoreToDisk (main.cu:974-989); -defocus of the parsed (negated) value
        const float defocus_print = (-1) * (-ctf.defocus);
        for (size_t k = 0; k < np; ++k) {
            const gs_pick& pk = picks[k];
            fprintf(fp, "%d\t%s\tdefocus=%f\tdfdiff=%f\tdfang=%f\teuler=%f,%f,%f\tcenter=%f,%f\tscore=%f\n", ent.nn,
                    ent.path.c_str(), defocus_print, ctf.dfdiff, ctf.dfang, eul.alt[pk.template_index],
                    eul.az[pk.template_index], pk.phi, pk.center_x, pk.center_y, pk.score);
        }
        gs_picks_free(picks);
        float ms[GS_TIMING_COUNT];
        gs_get_timings(ctx, ms, GS_TIMING_COUNT);
        printf("Image %d: %zu picks, %.1f ms (preprocess %.1f, template spectra %.1f, correlation %.1f)\n", n, np,
               ms[3], ms[0], ms[1], ms[2]);
        printf("------------------------Image %d finished--------------------------------\n", n);
    }
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    printf("Total consumed time is: %f seconds\n", secs);
    fclose(fp);
    gs_ctx_destroy(ctx);
    return 0;
}
