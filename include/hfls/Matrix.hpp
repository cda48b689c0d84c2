// Vector of the reference's surface (ostravaTokyo/hfls src/Matrix.hpp:244-254):
// a dense FP64 vector whose storage is the public member `dense`.  Outputs
// of the Cluster operators are resized on first use, as the reference does
// (get_numel() == 0 -> zero_dense, Cluster.cpp:1196-1199).
#ifndef HFLS_MATRIX_HPP
#define HFLS_MATRIX_HPP

#include <string>
#include <vector>

using namespace std;

class Vector {
public:
    Vector() {}
    vector<double> dense;
    void zero_dense(int n) { dense.assign(size_t(n > 0 ? n : 0), 0.0); }
    int get_numel() const { return int(dense.size()); }
    void set_label(const string &l) { label = l; }
    string get_label() const { return label; }
    void add(const Vector &b, double alpha) {           // this += alpha * b (Matrix::add)
        for (size_t i = 0; i < dense.size() && i < b.dense.size(); ++i) dense[i] += alpha * b.dense[i];
    }
    static double dot(const Vector &a, const Vector &b) {   // left-to-right sum (Matrix::dot)
        double s = 0.0;
        for (size_t i = 0; i < a.dense.size() && i < b.dense.size(); ++i) s += a.dense[i] * b.dense[i];
        return s;
    }

private:
    string label;
};

#endif
