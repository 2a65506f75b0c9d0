// Drives the learned-init pipeline through the C ABI from C++ (host buffers
// only, no CUDA headers): the way a C++ host of the align call would use it.
//
// Input file (little endian): int32 M, M x float[4] map; int32 L, L x
// (double resolution, step, max iterations, epsilon); int32 W, W floats of network weights;
// float[3] centre, float scale, float[6] delta scale; int32 B, (B + 1) int32
// offsets, offsets[B] x float[4] points, B x float[16] guesses.
// Output file: B x float[16] poses, B int32 converged, B double fitness,
// B int32 status, B int32 choice, B x float[16] starts.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ndt_b200.h"

namespace {

template <class T>
void get(FILE *f, T *p, size_t n) {
    if (std::fread(p, sizeof(T), n, f) != n) {
        std::fprintf(stderr, "short input file\n");
        std::exit(2);
    }
}

template <class T>
void put(FILE *f, const std::vector<T> &v) {
    if (std::fwrite(v.data(), sizeof(T), v.size(), f) != v.size()) std::exit(3);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input output\n", argv[0]);
        return 2;
    }
    FILE *in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int M = 0, L = 0, W = 0, B = 0;
    get(in, &M, 1);
    std::vector<float> map(4 * (size_t)M);
    get(in, map.data(), map.size());
    get(in, &L, 1);
    std::vector<double> lv(4 * (size_t)L);
    get(in, lv.data(), lv.size());
    get(in, &W, 1);
    std::vector<float> w(W);
    get(in, w.data(), w.size());
    float centre[3], scale, dscale[6];
    get(in, centre, 3);
    get(in, &scale, 1);
    get(in, dscale, 6);
    get(in, &B, 1);
    std::vector<int> offs(B + 1);
    get(in, offs.data(), offs.size());
    std::vector<float> pts(4 * (size_t)offs[B]), guesses(16 * (size_t)B);
    get(in, pts.data(), pts.size());
    get(in, guesses.data(), guesses.size());
    std::fclose(in);

    std::vector<ndt_ctx *> levels(L, nullptr);
    for (int l = 0; l < L; ++l) {
        ndt_params p;
        ndt_params_corrected(&p);
        p.resolution = (float)lv[4 * l];
        p.step_size = lv[4 * l + 1];
        p.max_iterations = (int)lv[4 * l + 2];
        p.transformation_epsilon = lv[4 * l + 3];
        if (ndt_create(&p, 0, &levels[l]) != NDT_OK) {
            std::fprintf(stderr, "ndt_create failed\n");
            return 4;
        }
        if (ndt_set_map(levels[l], map.data(), M) != NDT_OK) {
            std::fprintf(stderr, "ndt_set_map: %s\n", ndt_last_error(levels[l]));
            return 4;
        }
    }
    ndt_mlp *net = nullptr;
    if (ndt_mlp_create(0, &net) != NDT_OK || W != ndt_mlp_num_weights() ||
        ndt_mlp_set_input_frame(net, centre, scale, dscale) != NDT_OK || ndt_mlp_set_weights(net, w.data(), W) != NDT_OK) {
        std::fprintf(stderr, "network set-up failed\n");
        return 5;
    }
    ndt_learned_params lp;
    ndt_learned_params_default(&lp);
    std::vector<float> out(16 * (size_t)B), start(16 * (size_t)B);
    std::vector<int> conv(B), status(B), choice(B);
    std::vector<double> fit(B);
    int rc = ndt_align_batch_learned(net, levels.data(), L, &lp, B, pts.data(), offs.data(), guesses.data(),
                                     out.data(), conv.data(), fit.data(), status.data(), choice.data(), start.data());
    if (rc != NDT_OK) {
        std::fprintf(stderr, "ndt_align_batch_learned: %s\n", ndt_mlp_last_error(net));
        return 6;
    }
    int tc_error = 0;
    ndt_mlp_synchronize(net, &tc_error);
    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 3;
    put(o, out);
    put(o, conv);
    put(o, fit);
    put(o, status);
    put(o, choice);
    put(o, start);
    std::fclose(o);
    ndt_mlp_destroy(net);
    for (ndt_ctx *c : levels) ndt_destroy(c);
    std::printf("learned batch of %d through the C ABI: ok (tensor-core error flag %d)\n", B, tc_error);
    return tc_error ? 7 : 0;
}
