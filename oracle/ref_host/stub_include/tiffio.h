/* Declaration-only stand-in for libtiff (absent from this image).  The
 * reference headers mention the TIFF handle type; none of the classes the
 * checker compiles calls libtiff. */
#ifndef MC3_STUB_TIFFIO_H
#define MC3_STUB_TIFFIO_H
typedef struct tiff TIFF;
#endif
