/*
 * hpmc_types.h -- scalar types of HPMC's C API without any GL header.
 *
 * The reference API (hpmc/include/hpmc.h:289) takes its argument types from
 * <GL/glew.h>.  The B200 build has no GL on its path, so the same scalar
 * typedefs are declared here with the widths GL gives them.  If GL headers
 * were included first, theirs are used.
 */
#ifndef HPMC_B200_TYPES_H
#define HPMC_B200_TYPES_H

#if !defined(__gl_h_) && !defined(__GL_H__) && !defined(__glew_h__) && !defined(HPMC_ORACLE_SHIM_GLEW_H)
typedef int           GLint;
typedef int           GLsizei;
typedef unsigned int  GLuint;
typedef unsigned int  GLenum;
typedef float         GLfloat;
typedef unsigned char GLboolean;
#ifndef GL_FALSE
#define GL_FALSE 0
#endif
#ifndef GL_TRUE
#define GL_TRUE 1
#endif
#endif

#endif
