// monolish-compatible vector math used by the solve path
// (include/monolish/vml/monolish_vector_vml.hpp: sub, mul, reciprocal).
#pragma once
#include "monolish/common/monolish_common.hpp"

namespace monolish {
namespace vml {

void sub(const vector<double> &a, const vector<double> &b, vector<double> &y);
void sub(const vector<float> &a, const vector<float> &b, vector<float> &y);
void mul(const vector<double> &a, const vector<double> &b, vector<double> &y);
void mul(const vector<float> &a, const vector<float> &b, vector<float> &y);
void reciprocal(const vector<double> &a, vector<double> &y);
void reciprocal(const vector<float> &a, vector<float> &y);

}  // namespace vml
}  // namespace monolish
