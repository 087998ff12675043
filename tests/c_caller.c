/* A plain C caller of the library's C ABI (include/sgd_b200.h), the way a
 * C, cgo or FFI binding would call it.  Runs without a GPU: it exercises the
 * host-only geometry entry point and the error protocol (NULL / -1 plus
 * sgd_last_error(), never an exception across the ABI).  Built and run by
 * tests/test_c_caller.py; prints "ok" and exits 0 when every check holds. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "sgd_b200.h"

static int failures = 0;

static void expect(int cond, const char* what) {
    if (!cond) {
        printf("FAILED: %s (last error: %s)\n", what, sgd_last_error() ? sgd_last_error() : "(null)");
        ++failures;
    }
}

static int has(const char* needle) {
    const char* e = sgd_last_error();
    return e && strstr(e, needle) != NULL;
}

int main(void) {
    double ang[4] = {0.0, 0.5, 1.0, 1.5};
    double pm[48];
    float pmi[48];
    double b[48], x[64];
    void* h;

    /* host-only: the index-space projection matrices of four views */
    expect(sgd_geometry_pmi(8, 8, 1, 4, 12, 1, 1.0, 1.0, 1.0, 1.0, 1.0, 40.0, 20.0, ang, NULL, NULL, pm, pmi) == 0,
           "sgd_geometry_pmi succeeds on the host");
    expect(isfinite(pmi[0]) && isfinite(pmi[47]) && pmi[11] != 0.0f, "pmi is finite");

    /* bad geometry: NULL and the reason, for the reference's constructors */
    h = b1_init(8, 8, 4, 12, 1.0, 1.0, 1.0, 10.0, 20.0, ang, NULL, NULL);
    expect(h == NULL && has("lso < lsd"), "b1_init rejects lsd < lso");
    h = b0_init(0, 8, 4, 12, 1.0, 1.0, 1.0, 40.0, 20.0, ang, NULL, NULL);
    expect(h == NULL && has("invalid sizes"), "b0_init rejects nx = 0");
    h = SF_init(8, 8, 4, 12, 1.0, -1.0, 1.0, 40.0, 20.0, ang);
    expect(h == NULL && has("pitches"), "SF_init rejects a negative pitch");
    h = h0_init(8, 8, 4, 12, 0.0, 1.0, 40.0, 20.0, ang, NULL, NULL);
    expect(h == NULL && has("pitches"), "h0_init rejects dt = 0");
    h = b1_3d_init(8, 8, 8, 4, 12, 12, 1.0, 1.0, 1.0, 1.0, 0.0, 40.0, 20.0, ang);
    expect(h == NULL && has("pitches"), "b1_3d_init rejects dv = 0");
    ang[1] = NAN;
    h = hl_init(8, 8, 4, 12, 1.0, 1.0, 40.0, 20.0, ang, NULL, NULL);
    expect(h == NULL && has("angle of view 1"), "hl_init rejects a NaN angle");
    ang[1] = 0.5;

    /* calls on a NULL layer: -1 / nothing, with the reason */
    expect(b1_forward_projection(b, x, NULL) == -1 && has("null"), "b1_forward_projection(NULL layer) = -1");
    expect(sgd_b1_backward_projection(b, x, NULL) == -1 && has("null"), "sgd_b1_backward_projection(NULL) = -1");
    b1_backward_projection(b, x, NULL); /* void: must return, not abort */
    expect(has("null"), "b1_backward_projection(NULL layer) records the error");
    expect(SF_forward_projection(b, x, NULL) == -1, "SF_forward_projection(NULL layer) = -1");
    b1_destroy(NULL); /* freeing nothing is a no-op */

    /* the reference's generator with a buffer it cannot fill: -1 */
    expect(pixel_matrix_generation(4, 12, 8, 8, 1.0, 1.0, 1.0, 40.0, 20.0, NULL, 10) == -1,
           "pixel_matrix_generation(NULL buffer) = -1");

    if (failures) return 1;
    printf("ok\n");
    return 0;
}
