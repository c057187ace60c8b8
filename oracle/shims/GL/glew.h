/*
 * Compile-only stand-in for <GL/glew.h>, project-written.  The reference's
 * headers name the type GLuint, and meshless_vis/meshless_vis_cpu.cpp:236-248
 * (vis_opengl_fourier_volume_rendering) names three buffer calls.  There is no
 * graphics stack here: the type is an unsigned int and the three calls expand
 * to expressions that do nothing.  Nothing in the tests or the bench calls the
 * OpenGL entry point of the reference build.
 */
#ifndef MV_SHIM_GLEW_H
#define MV_SHIM_GLEW_H

typedef unsigned int GLuint;
typedef unsigned int GLenum;

#define GL_PIXEL_UNPACK_BUFFER 0x88EC
#define GL_WRITE_ONLY 0x88B9

#define glBindBuffer(target, buffer) ((void)(target), (void)(buffer))
#define glMapBuffer(target, access) ((void)(target), (void)(access), (void*)0)
#define glUnmapBuffer(target) ((void)(target), 1)

#endif
