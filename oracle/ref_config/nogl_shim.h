/* Force-included only when compiling the reference's opengl2.c for the test
 * oracle. With OpenGL disabled every drawing routine in that file is compiled
 * out except one, which still names two GL calls; these no-op stand-ins let
 * the file compile. Nothing is drawn: graphics are unavailable on this box. */
#ifndef SMOLDYN_ORACLE_NOGL_SHIM_H
#define SMOLDYN_ORACLE_NOGL_SHIM_H
typedef double GLdouble;
#define glRasterPos3d(x, y, z) ((void)0)
#define glutBitmapCharacter(font, c) ((void)(font), (void)(c))
#endif
