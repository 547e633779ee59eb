#ifndef Xyce_N_LAS_Vector_h
#define Xyce_N_LAS_Vector_h
#include <vector>
#include <N_LAS_fwd.h>
class N_LAS_Vector {
public:
  explicit N_LAS_Vector(int n = 0) : v_(n, 0.0) {}
  double & operator[](int i) { return v_[i]; }
  const double & operator[](int i) const { return v_[i]; }
  std::vector<double> & data() { return v_; }
  void putScalar(double s) { for (auto & x : v_) x = s; }
private:
  std::vector<double> v_;
};
#endif
