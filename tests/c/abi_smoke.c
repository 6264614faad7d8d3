/* A C caller of libvoxrt that needs no GPU: compiled as strict C99 against
 * include/voxrt.h, it exercises the host-only entry points (constants,
 * camera, host world, ray-query wire codec) and the error reporting. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "voxrt.h"

#define CHECK(c)                                                     \
    do {                                                             \
        if (!(c)) {                                                  \
            fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
            return 1;                                                \
        }                                                            \
    } while (0)

int main(void) {
    VxTraceParams p;
    VxCamera cam;
    VxHostWorld *hw = NULL;
    VxBrick *bricks = NULL;
    uint64_t *tm = NULL, *cm = NULL, *l4 = NULL;
    uint8_t *bu = NULL, *tu = NULL;
    const float pos[3] = {256.0f, 140.0f, 256.0f};
    const int32_t zero[3] = {0, 0, 0};
    VxRay rays[2];
    VxRay back[2];
    uint8_t frame[128];
    size_t len = 0, n = 0;
    uint64_t id = 0;

    CHECK(vx_abi_version() == VX_ABI_VERSION);
    CHECK(vx_default_params(&p) == VX_OK);
    CHECK(p.max_dist == 700.0f && p.max_iters == 1024 && p.any_max_iters == 768);
    CHECK(vx_camera_from_pose(pos, 0.0f, -0.26f, 1.2217305f, 640, 360, zero, &cam) == VX_OK);
    CHECK(fabsf(cam.forward[0] * cam.forward[0] + cam.forward[1] * cam.forward[1] +
                cam.forward[2] * cam.forward[2] - 1.0f) < 1e-5f);

    /* host mirror of the world: one voxel set, dirty tracking, masks */
    CHECK(vx_host_world_create(64, 16, 64, &hw) == VX_OK);
    CHECK(vx_host_world_arrays(hw, &bricks, &tm, &cm, &l4, &bu, &tu) == VX_OK);
    /* a new world starts all dirty (its first sync is a full upload) */
    CHECK(vx_host_world_dirty_count(hw) == 64 * 16 * 64);
    CHECK(vx_host_world_set_voxel(hw, 5, 6, 7, 4) >= 0);
    CHECK(bricks[1 + 1 * 64 + 1 * 64 * 16].occupancy != 0);
    CHECK(vx_host_world_rebuild(hw) == VX_OK);
    CHECK(cm[0] != 0 && l4[0] != 0);
    CHECK(vx_host_world_destroy(hw) == VX_OK);

    /* wire codec round trip */
    memset(rays, 0, sizeof(rays));
    rays[0].org[0] = 1.5f; rays[0].dir[1] = -1.0f; rays[0].tmax = 64.0f; rays[0].kind = 1;
    rays[1].org[2] = -3.0f; rays[1].dir[0] = 1.0f; rays[1].tmax = 700.0f;
    CHECK(vx_wire_query_bytes(2) == 24 + 2 * 32);
    CHECK(vx_wire_encode_query(9, rays, 2, frame, sizeof(frame), &len) == VX_OK);
    CHECK(len == vx_wire_query_bytes(2));
    CHECK(vx_wire_decode_query(frame, len, &id, back, 2, &n) == VX_OK);
    CHECK(id == 9 && n == 2 && memcmp(rays, back, sizeof(rays)) == 0);
    CHECK(vx_wire_decode_query(frame, len - 1, &id, back, 2, &n) == VX_ERR_INVALID);
    CHECK(strlen(vx_last_error()) > 0);

    /* invalid arguments fail with a status, never abort */
    CHECK(vx_world_create(NULL, NULL) == VX_ERR_INVALID);
    CHECK(vx_render_primary(NULL, &cam, &p, NULL, NULL, NULL) == VX_ERR_INVALID);
    printf("c abi ok\n");
    return 0;
}
