// Test infrastructure: the reference's own near-interface dump, Write_txt
// (src/helper.h:442-575), called by the harness (--write-txt).  It lives in
// a translation unit of its own because helper.h brings in every plugin
// header of the reference.  Write_txt writes "Numerical Solutions.txt" and
// "Numerical Error.txt" into the working directory and supports the
// reference's Eq_0..Eq_7 only.
#include <fstream>
#include <iostream>
#include <string>

// helper.h expects what src/main.cc has in scope before it
using namespace std;
#include "helper.h"

void ref_write_txt(Intersections& inter, Mesh& mesh, Beta& beta, CubicDoub& uh, int equation, double t) {
  Write_txt(inter, mesh, beta, uh, equation, t);
}
