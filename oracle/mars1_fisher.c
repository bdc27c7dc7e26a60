/* Test infrastructure only: a harness around the reference's own 1998 C Fisher classifier
 * (reference/mars1/index_func.c: FisherIndexing, newclass, variance_class, contraction;
 * coding_func.c: flips), compiled from the reference's sources by `make -C oracle ref` into
 * oracle/_ref/libmars1_fisher.so.  It pins the classified search's bucketing: the tests
 * compare the oracle's restatement (crates/mars-search/src/classify.rs) and the device's
 * buckets with what the reference's C code computes on the same planes.  Nothing in the
 * library links or loads it.
 *
 * The reference's contraction() bounds its column index by the image height
 * (index_func.c:186-207), so only square planes give the intended contraction; the tests
 * use square planes. */
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#include <fcntl.h>

#define EXTERN
#include "globals.h"
#include "prot.h"

/* FisherIndexing prints progress on stdout: silence it for the call. */
static int quiet_begin(void) {
    int saved, devnull;
    fflush(stdout);
    saved = dup(1);
    devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) {
        dup2(devnull, 1);
        close(devnull);
    }
    return saved;
}

static void quiet_end(int saved) {
    fflush(stdout);
    if (saved >= 0) {
        dup2(saved, 1);
        close(saved);
    }
}

/* Classifies every domain position of one (size, shift) level of a w x h plane with the
 * reference's own code: the contraction, then per position the window FisherIndexing reads
 * (index_func.c:649-690) through newclass, flips and variance_class.  Outputs, per
 * position in raster order (row-major over the ((h - 2 size) / shift + 1) x
 * ((w - 2 size) / shift + 1) grid): bucket = class * 24 + variance class, and the
 * canonicalising isometry; counts[72]: positions per bucket; first_nonempty: the bucket
 * FisherIndexing copies into every empty one.  FisherIndexing itself is run on the same
 * plane and its lists checked against these: a non-empty bucket's list has counts[bucket]
 * nodes, each at a position classified into that bucket with the same isometry, and every
 * empty bucket holds the first non-empty bucket's list.  Returns 0, -1 on bad arguments,
 * -2 when the lists disagree. */
int m1_fisher_domains(const unsigned char *px, int w, int h, int size, int shift,
                      unsigned char *bucket, unsigned char *iso, unsigned int *counts,
                      int *first_nonempty) {
    int i, j, k, v, x, y, ncol, nrow, saved, first = -1, bad = 0;
    PIXEL **rows;
    double **domi, **flip;
    if (!px || !bucket || !iso || !counts || size < 2 || shift < 1 || w < 2 * size ||
        h < 2 * size)
        return -1;
    image_width = w;
    image_height = h;
    SHIFT = shift;
    rows = (PIXEL **)malloc(sizeof(PIXEL *) * h);
    for (i = 0; i < h; ++i) rows[i] = (PIXEL *)(px + (size_t)i * w);
    matrix_allocate(contract, w / 2, h / 2, double)
    contraction(contract, rows, 0, 0);

    ncol = (w - 2 * size) / shift + 1;
    nrow = (h - 2 * size) / shift + 1;
    memset(counts, 0, 72 * sizeof(unsigned int));
    matrix_allocate(domi, size, size, double)
    matrix_allocate(flip, size, size, double)
    for (i = 0; i < nrow; ++i)
        for (j = 0; j < ncol; ++j) {
            const int r = i * shift, c = j * shift;
            int is, clas, var;
            for (x = 0; x < size; ++x)
                for (y = 0; y < size; ++y) domi[x][y] = contract[x + (r >> 1)][y + (c >> 1)];
            newclass(size, domi, &is, &clas);
            flips(size, domi, flip, is);
            var = variance_class(size, flip);
            bucket[(size_t)i * ncol + j] = (unsigned char)(clas * 24 + var);
            iso[(size_t)i * ncol + j] = (unsigned char)is;
            counts[clas * 24 + var]++;
        }
    for (k = 0; k < 72 && first < 0; ++k)
        if (counts[k]) first = k;

    /* FisherIndexing's own lists. */
    for (k = 0; k < 3; ++k)
        for (v = 0; v < 24; ++v) class_fisher[0][k][v] = NULL;
    saved = quiet_begin();
    FisherIndexing(size, 0);
    quiet_end(saved);
    for (k = 0; k < 3; ++k)
        for (v = 0; v < 24; ++v) {
            const int key = k * 24 + v;
            struct c *p = class_fisher[0][k][v];
            unsigned int len = 0;
            if (!counts[key]) {
                if (p != class_fisher[0][first / 24][first % 24]) bad = 1;
                continue;
            }
            for (; p; p = p->next, ++len) {
                const size_t pos = (size_t)(p->ptr_x / shift) * ncol + (size_t)(p->ptr_y / shift);
                if (bucket[pos] != key || iso[pos] != p->iso) bad = 1;
            }
            if (len != counts[key]) bad = 1;
        }
    if (first_nonempty) *first_nonempty = first;
    free(domi[0]);
    free(domi);
    free(flip[0]);
    free(flip);
    free(contract[0]);
    free(contract);
    contract = NULL;
    free(rows);
    return bad ? -2 : 0;
}

/* The range side of FisherCoding (coding_func.c:228-241): class, variance class and
 * canonicalising isometry of the size x size block at (row, col) of a plane of stride w. */
int m1_fisher_range(const unsigned char *px, int w, int size, int row, int col, int *clas,
                    int *var_class, int *isom) {
    int x, y;
    double **blk, **flip;
    if (!px || size < 2 || !clas || !var_class || !isom) return -1;
    matrix_allocate(blk, size, size, double)
    matrix_allocate(flip, size, size, double)
    for (x = 0; x < size; ++x)
        for (y = 0; y < size; ++y) blk[x][y] = (double)px[(size_t)(row + x) * w + col + y];
    newclass(size, blk, isom, clas);
    flips(size, blk, flip, *isom);
    *var_class = variance_class(size, flip);
    free(blk[0]);
    free(blk);
    free(flip[0]);
    free(flip);
    return 0;
}
