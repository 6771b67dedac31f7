/*
 * The reference's Viewer (viewer.h) with output switched off: the same class, whose View_*
 * calls write nothing.  Controller::solve writes VTK snapshots through it at start, every
 * WriteInterval steps and at the end (controller.cpp:86, 122-131, 226-227); a run that only
 * wants the particles links this in place of viewer.cpp.  Snapshots in the reference's
 * format are available from apcloud.vtk on the Python side.
 */
#include <cstring>

#include "viewer.h"

Viewer::Viewer(Physical_particle *physical_particle1, Computational_particle *computational_particle1)
    : pp(physical_particle1), cp(computational_particle1) {
  file_p = nullptr;
  file_c = nullptr;
  file_name_p[0] = file_name_c[0] = '\0';
}

void Viewer::View_Physical_Particles(double) {}
void Viewer::View_Physical_Particles_Limit(double, double, double, double, double, double, double) {}
void Viewer::View_Computational_Particles(double) {}
