/*
 * Types-only stand-in for <GL/glew.h>, used ONLY to compile the three
 * reference source files that make no GL calls (hpmc/src/init.cpp,
 * hpmc/src/tables.cpp, hpmc/src/shadergen.cpp) into the test oracle under
 * oracle/_ref/.  It declares the scalar GL typedefs those files name and
 * nothing else: no GL function, no loader, no rendering.
 *
 * Test infrastructure only; the product never includes this header.
 */
#ifndef HPMC_ORACLE_SHIM_GLEW_H
#define HPMC_ORACLE_SHIM_GLEW_H

typedef int           GLint;
typedef int           GLsizei;
typedef unsigned int  GLuint;
typedef unsigned int  GLenum;
typedef float         GLfloat;
typedef unsigned char GLboolean;

#define GL_FALSE 0
#define GL_TRUE  1

#endif
