// No graphics stack: the drawing calls in the reference's surface class become no-ops.
#pragma once
#define glBegin(...) ((void)0)
#define glEnd(...) ((void)0)
#define glNormal3d(...) ((void)0)
#define glNormal3dv(...) ((void)0)
#define glNormal3f(...) ((void)0)
#define glNormal3fv(...) ((void)0)
#define glPopMatrix(...) ((void)0)
#define glPushMatrix(...) ((void)0)
#define glTexCoord2d(...) ((void)0)
#define glTexCoord2f(...) ((void)0)
#define glTranslatef(...) ((void)0)
#define glVertex3d(...) ((void)0)
#define glVertex3dv(...) ((void)0)
#define glVertex3f(...) ((void)0)
#define glVertex3fv(...) ((void)0)
#define GL_LINE 1
#define GL_LINES 2
#define GL_POINTS 3
#define GL_TRIANGLES 4
