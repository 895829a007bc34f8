/* A plain C99 caller of the extended ABI (include/ceemdan_b200.h), built by tests/test_abi.py
 * with gcc -std=c99 -pedantic -Werror and linked against libceemdan_b200.so alone.  It makes
 * only calls that the library rejects on the host (no device is touched) and prints their
 * status codes. */
#include <stdio.h>

#include "ceemdan_b200.h"

int main(void) {
    ceemdan_options o;
    ceemdan_tape* t = NULL;
    ceemdan_default_options(&o);
    printf("%d %d %d %d %d %lu %d\n",
           (int)ceemdan_plain_f64(0, 100, 5, 10, NULL, NULL, NULL, 0.2, &o, NULL),
           (int)ceemdan_forward_taped_f64(4, 100, 5, 10, NULL, NULL, NULL, 0.2, &o, NULL, NULL),
           (int)ceemdan_forward_checkpointed_f64(4, 100, 5, 10, NULL, NULL, NULL, 0.2, &o, NULL,
                                                 &t),
           (int)ceemdan_backward_f64(NULL, NULL, NULL, NULL),
           t == NULL, (unsigned long)ceemdan_tape_bytes(t), ceemdan_tape_iterations(t, 0));
    ceemdan_tape_free(t);
    return 0;
}
