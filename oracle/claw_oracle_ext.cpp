// ORACLE — test infrastructure only (see claw_oracle.cpp header).
// Extension point for the 2D Euler (Roe) solver and the 3D path.
namespace orc_ext {
typedef void (*rpn2_t)(int, int, int, int, int, int, int, const double*, const double*,
                       const double*, const double*, double*, double*, double*, double*);
typedef void (*rpt2_t)(int, int, int, int, int, int, int, int, const double*, const double*,
                       const double*, const double*, const double*, const double*, double*,
                       double*);
bool pick2_ext(int, rpn2_t*, rpt2_t*) { return false; }
}  // namespace orc_ext
