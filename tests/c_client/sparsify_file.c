/* A plain-C client of libspecspars.so: what a Rust (or any FFI) caller of the path does, with no Python in
 * between.  Reads a graph from a Matrix Market file, derives the CLI parameters (sparsify_dataset, lib.rs:149-156),
 * sparsifies it on device 0 and writes L_H.
 *
 *   sparsify_file <in.mtx> <out.mtx>
 *
 * Exit status: 0 done; 3 no CUDA device (the library's clean error); 1 any other failure. */
#include <stdio.h>

#include "specspars.h"

static int failed(const char* what, int rc) {
    fprintf(stderr, "%s failed (%d): %s\n", what, rc, ssp_last_error());
    return 1;
}

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <in.mtx> <out.mtx>\n", argv[0]);
        return 1;
    }
    ssp_csc_out g;
    int rc = ssp_read_mtx(argv[1], &g);
    if (rc != SSP_OK) return failed("ssp_read_mtx", rc);
    ssp_params p;
    ssp_params_cli(&p, 0.5, 0, 0, 0, 0, NULL);
    printf("n %lld nnz %lld jl_dim %d\n", (long long)g.n, (long long)g.nnz, ssp_params_jl_dim(&p, g.n));

    ssp_context* ctx = NULL;
    rc = ssp_context_create(0, &ctx);
    if (rc == SSP_ERR_NO_DEVICE) {
        printf("no device: %s\n", ssp_last_error());
        ssp_csc_free(&g);
        return 3;
    }
    if (rc != SSP_OK) return failed("ssp_context_create", rc);

    const ssp_csc in = {g.n, g.nnz, g.colptr, g.rowidx, g.values, SSP_MEM_HOST};
    ssp_csc_out h;
    ssp_stats st;
    rc = ssp_sparsify(ctx, &in, &p, SSP_MEM_HOST, &h, &st);
    if (rc != SSP_OK) return failed("ssp_sparsify", rc);
    const ssp_csc out = {h.n, h.nnz, h.colptr, h.rowidx, h.values, SSP_MEM_HOST};
    rc = ssp_write_mtx(argv[2], &out);
    if (rc != SSP_OK) return failed("ssp_write_mtx", rc);
    printf("m_in %lld m_out %lld\n", (long long)st.m_in, (long long)st.m_out);
    ssp_csc_free(&h);
    ssp_csc_free(&g);
    ssp_context_destroy(ctx);
    return 0;
}
