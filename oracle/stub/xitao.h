/* Empty stand-in for the XiTAO runtime header, which the reference's
 * 3d/traverse_eager.h includes unconditionally.  The OpenMP path that the
 * oracle builds (no USE_XITAO) uses nothing from it. */
