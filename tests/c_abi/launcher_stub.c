/* A reference-style launcher fragment in plain C against include/xmcml_b200.h: parse the model files,
 * allocate the output, check the specular reflectance and the layout table, and (when asked) run the
 * LaunchOMP replacement. Compiled and run by tests/test_c_abi.py; the run step needs a GPU. */
#include <stdio.h>
#include <string.h>

#include "xmcml_b200.h"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    InputInfo in;
    OutputInfo out;
    memset(&in, 0, sizeof(in));
    memset(&out, 0, sizeof(out));
    if (!xmc_parse_input_file(argv[1], &in) || !xmc_parse_surface_file(argv[2], &in)) {
        fprintf(stderr, "parse: %s\n", xmc_last_error());
        return 3;
    }
    xmc_init_output(&in, &out);
    printf("version %d layers %d surfaces %d detectors %d grid %d rsp %.12f\n", xmc_version(), in.numberOfLayers,
           in.numberOfSurfaces, out.numberOfDetectors, out.gridSize, xmc_specular_reflectance(in.layerInfo));
    int64_t offs[256];
    printf("layout fields %d\n", xmc_layout_offsets(offs, 256));
    int rc = 0;
    if (argc > 3 && strcmp(argv[3], "--run") == 0) {
        MCG59 rng;
        rng.value = 2 * 777 + 1;
        rng.offset = 302875106592253ULL;
        rc = xmc_launch_omp(&in, &out, &rng, 0);
        double w = 0.0;
        for (int d = 0; d < out.numberOfDetectors; ++d) w += out.detectorInfo[d].weight;
        printf("run status %d detected weight %.6f\n", rc, w);
        xmc_launch_release();
    }
    xmc_free_output(&out);
    xmc_free_input(&in);
    return rc == XMC_OK || rc == XMC_ERR_BUDGET ? 0 : 4;
}
