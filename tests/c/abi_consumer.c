/* A plain C99 consumer of include/rtm.h, as a MEX gateway or any other C caller sees it. It calls only
 * the entry points that need no GPU and prints one result per line for tests/test_c_consumer.py. */
#include <stdio.h>
#include <string.h>

#include "rtm.h"

static void print_error(const char* what, int status) {
    char msg[256];
    rtm_last_error(msg, sizeof msg);
    printf("%s %d %s\n", what, status, msg);
}

int main(void) {
    int major = 0, minor = 0, patch = 0;
    double est[6], scratch = 0, gap[2 * 17];
    int64_t port[3] = {1, 4, 10};
    double dir[3] = {0, 0, -1}, pol[3] = {1, 0, 0}, one = 1, sink[2];
    int i, status;

    status = rtm_version(&major, &minor, &patch);
    printf("version %d %d.%d.%d\n", status, major, minor, patch);

    status = rtm_estimate_bytes(256, 256, RTM_PRODUCT_SPLIT, RTM_METHOD_GMRES, 1, 50, 1000, est);
    printf("estimate %d", status);
    for (i = 0; i < 6; ++i) printf(" %.17g", est[i]);
    printf("\n");

    status = rtm_fixed_scratch_bytes(&scratch);
    printf("scratch %d %.17g\n", status, scratch);

    /* a 4 x 3 plate of 0.1 x 0.2 faces: 9 x-directed rooftops (edges 0.2), then 8 y-directed (edges 0.1) */
    memset(gap, 0, sizeof gap);
    status = rtm_delta_gap(4, 3, 0.1, 0.2, port, 3, 0, 3.0, gap, RTM_HOST);
    printf("gap %d", status);
    for (i = 0; i < 17; ++i) printf(" %.17g", gap[2 * i]);
    printf("\n");

    status = rtm_delta_gap(4, 3, 0.1, 0.2, port, 3, 0, 3.0, NULL, RTM_HOST);
    print_error("null", status);
    status = rtm_plane_wave(8, 8, 0.05, 0.05, 8, 6.283185307179586, dir, pol, &one, 70000, sink, RTM_HOST, NULL);
    print_error("rhs", status);

    /* the serving loop: a request above the whole budget fails at submission, before any device work */
    {
        rtm_server_config cfg;
        rtm_server* srv = NULL;
        rtm_request req;
        rtm_request_result res;
        uint64_t id = 0;
        memset(&cfg, 0, sizeof cfg);
        cfg.budget_bytes = 1e6;
        cfg.max_active = 2;
        cfg.precision = RTM_FP64;
        memset(&req, 0, sizeof req);
        req.count_x = 40;
        req.count_y = 32;
        req.size_x = req.size_y = 0.05;
        req.wavenumber = 6.283185307179586;
        req.excitation = RTM_EXCITE_PLANE_WAVE;
        req.direction[2] = -1;
        req.polarization[0] = 1;
        req.method = RTM_METHOD_GMRES;
        req.preconditioner = 1;
        req.tolerance = 1e-6;
        req.max_iterations = 1000;
        req.restart = 50;
        status = rtm_server_create(&cfg, &srv);
        printf("server_create %d\n", status);
        status = rtm_server_submit(srv, &req, &id);
        printf("server_submit %d %llu\n", status, (unsigned long long)id);
        memset(&res, 0, sizeof res);
        status = rtm_server_poll(srv, id, 0, &res, NULL, 0, 1);
        printf("server_poll %d %d %d %.17g\n", status, res.state, res.status, res.bytes);
        status = rtm_server_destroy(srv);
        printf("server_destroy %d\n", status);
    }
    return 0;
}
