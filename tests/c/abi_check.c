/* A C host against include/genesis_b200_mpm.h: calls the entry points that need no GPU
 * (version, struct sizes, capacity, workspace sizing, argument checks) and prints one
 * line per check; exit status 0 when every check holds. */
#include <stdio.h>
#include "genesis_b200_mpm.h"

#define CHECK(cond, what)                                          \
    do {                                                           \
        if (!(cond)) {                                             \
            printf("FAIL %s\n", what);                             \
            return 1;                                              \
        }                                                          \
        printf("ok %s\n", what);                                   \
    } while (0)

int main(void) {
    int32_t sizes[7];
    CHECK(mpm_abi_version() == MPM_ABI_VERSION, "abi version");
    CHECK(mpm_struct_sizes(sizes) == MPM_OK, "struct sizes call");
    CHECK(sizes[0] == (int32_t)sizeof(mpm_instance) && sizes[1] == (int32_t)sizeof(mpm_material) &&
              sizes[2] == (int32_t)sizeof(mpm_problem) && sizes[3] == (int32_t)sizeof(mpm_particles) &&
              sizes[4] == (int32_t)sizeof(mpm_tables) && sizes[5] == (int32_t)sizeof(mpm_collider) &&
              sizes[6] == (int32_t)sizeof(mpm_force_field),
          "struct layout seen from C");
    int32_t max_chunks = 0;
    CHECK(mpm_max_chunks(100000, 4913, 128, &max_chunks) == MPM_OK && max_chunks >= 100000 / 128, "max chunks");
    mpm_problem prob = {1, 100000, 4913, 1, 128, max_chunks, 0, 0};
    uint64_t bytes = 0;
    CHECK(mpm_workspace_bytes(&prob, &bytes) == MPM_OK && bytes > 0, "workspace bytes");
    CHECK(bytes <= MPM_NOALLOC_SCRATCH_BYTES, "65^3 grid with 100k particles fits the no-alloc scratch");
    CHECK(mpm_workspace_bytes(NULL, &bytes) == MPM_E_INVALID, "null problem refused");
    mpm_problem bad = prob;
    bad.chunk_particles = 100;
    CHECK(mpm_workspace_bytes(&bad, &bytes) == MPM_E_INVALID, "chunk size must be 128, 256 or 512");
    return 0;
}
