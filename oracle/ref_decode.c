/*
 * Test infrastructure only: decodes a compressed (Gadget-encoded) particle
 * file with the reference's own functions -- readCompressedParticles and
 * decodeCompressedParticle (src/Gadget/BufVector3D.c), initGadgetDecodeParams
 * (src/Gadget/GadgetHeader.c), initGadId (src/Gadget/GadId.c) -- called the
 * way constructIndexWithSameThreadPool calls them (src/astr_rcount/main.c:
 * 739-763, one tile), and writes the float x,y,z of every particle to stdout.
 * Built by oracle/Makefile (target ref) against the reference's sources in
 * place; its output pins the oracle's and the GPU's decode.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "Gadget/BufVector3D.h"
#include "Gadget/GadId.h"
#include "Gadget/GadgetHeader.h"

int main(int argc, char *argv[])
{
    BufUshortVector3D *buv;
    GadgetHeader hdr;
    GadgetDecodeParams dparams;
    GadId idsys;
    unsigned long long n;
    if (argc != 2) {
        fprintf(stderr, "usage: %s compressed_file\n", argv[0]);
        return 2;
    }
    buv = constructBufUshortVector3D();
    buv = readCompressedParticles(buv, argv[1], &hdr);
    if (buv == NULL)
        return 1;
    initGadgetDecodeParams(&dparams, &hdr, 1);
    initGadId(&idsys, 1, dparams.nparticles_partile);
    for (n = 0; n < buv->nuvs; n++) {
        float pos[4];
        decodeCompressedParticle(getVectorBufUshortVector3D(buv, n), pos, &hdr, &idsys, n + dparams.id_start,
                                 dparams.cell_interval, dparams.unitsep);
        fwrite(pos, sizeof(float), 3, stdout);
    }
    destructBufUshortVector3D(buv);
    return 0;
}
