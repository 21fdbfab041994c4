/*
 * Test-oracle write_map (declared in mappraiser/include/mappraiser/iofiles.h):
 * writes the 12*nside^2 map values raw instead of as a HEALPix FITS table.
 * NOT product code.
 */
#include "fitsio.h"

#include <stdio.h>

void write_map(void *signal, int type, long nside, const char *filename, char nest, const char *coordsys) {
    (void) nest;
    (void) coordsys;
    long  npix = 12L * nside * nside;
    FILE *f    = fopen(filename, "wb");
    if (!f) {
        fprintf(stderr, "shim write_map: cannot open %s\n", filename);
        return;
    }
    fwrite(signal, type == TINT ? sizeof(int) : sizeof(double), (size_t) npix, f);
    fclose(f);
}
