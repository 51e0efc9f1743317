// Sauter-Schwab quadrature points of the near-field panel pairs (coincident,
// common-edge, common-vertex), shared by the assembly kernels and the shape
// adjoint.  For one 4D Gauss point (xsi, eta1, eta2, eta3) of the collapsed
// 4-cube with product weight `weight` (Gauss weights x 2A_x x 2A_y), every
// region of the relation calls
//   add(r1x, r2x, r1y, r2y, w, second, px1, px2, py1, py2)
// with the reference-triangle parameters of the point on each panel, the
// region's weight (Duffy Jacobian included), the swapped-argument flag of the
// coincide rule, and the parameters at which the basis functions are taken
// (the reference evaluates the swapped coincide term's bases at the unswapped
// points, `quirk`).  The maps follow single_layer_3d.py:178-367 and
// m_mats_coincide (BEM_manager.py:141-165).
#pragma once

#include "bem_internal.cuh"

template <class F>
__device__ __forceinline__ void near_points(int rel, bool quirk, double xsi, double eta1, double eta2, double eta3,
                                            double weight, F&& add) {
    if (rel == REL_COINCIDE) {
        const double jac = xsi * xsi * xsi * eta1 * eta1 * eta2;
        const double w0 = xsi, w1 = xsi * eta1, w2 = xsi * eta1 * eta2, w3 = xsi * eta1 * eta2 * eta3;
        // m_mats_coincide (BEM_manager.py:141-165) applied to w
        double z[3][4] = {{w0, w0 - w1 + w2, w3, w2},
                          {w0, w1 - w2 + w3, w2, w3},
                          {w0 - w3, w1 - w3, -w3, w2 - w3}};
        for (int m = 0; m < 3; ++m) {
            double r1x = z[m][0], r2x = z[m][1], r1y = z[m][0] - z[m][2], r2y = z[m][1] - z[m][3];
            add(r1x, r2x, r1y, r2y, weight * jac, false, r1x, r2x, r1y, r2y);
            if (quirk)
                add(r1x, r2x, r1y, r2y, weight * jac, true, r1x, r2x, r1y, r2y);
            else
                add(r1x, r2x, r1y, r2y, weight * jac, true, r1y, r2y, r1x, r2x);
        }
    } else if (rel == REL_VERTEX) {
        const double jac = xsi * xsi * xsi * eta2;
        add(xsi, xsi * eta1, xsi * eta2, xsi * eta2 * eta3, weight * jac, false, xsi, xsi * eta1, xsi * eta2,
            xsi * eta2 * eta3);
        add(xsi * eta2, xsi * eta2 * eta3, xsi, xsi * eta1, weight * jac, false, xsi * eta2, xsi * eta2 * eta3,
            xsi, xsi * eta1);
    } else {  // REL_EDGE
        double w0, w1, w2, w3;
        const double jac1 = xsi * xsi * xsi * eta1 * eta1;
        const double jac = jac1 * eta2;
        w0 = xsi; w1 = -xsi * eta1 * eta2; w2 = xsi * eta1 * (1.0 - eta2); w3 = xsi * eta1 * eta3;
        add(w0, w3, w0 + w1, w2, weight * jac1, false, w0, w3, w0 + w1, w2);
        w0 = xsi; w1 = -xsi * eta1 * eta2 * eta3; w2 = xsi * eta1 * eta2 * (1.0 - eta3); w3 = xsi * eta1;
        add(w0, w3, w0 + w1, w2, weight * jac, false, w0, w3, w0 + w1, w2);
        w0 = xsi * (1.0 - eta1 * eta2); w1 = xsi * eta1 * eta2; w2 = xsi * eta1 * eta2 * eta3;
        w3 = xsi * eta1 * (1.0 - eta2);
        add(w0, w3, w0 + w1, w2, weight * jac, false, w0, w3, w0 + w1, w2);
        w0 = xsi * (1.0 - eta1 * eta2 * eta3); w1 = xsi * eta1 * eta2 * eta3; w2 = xsi * eta1;
        w3 = xsi * eta1 * eta2 * (1.0 - eta3);
        add(w0, w3, w0 + w1, w2, weight * jac, false, w0, w3, w0 + w1, w2);
        w0 = xsi * (1.0 - eta1 * eta2 * eta3); w1 = xsi * eta1 * eta2 * eta3; w2 = xsi * eta1 * eta2;
        w3 = xsi * eta1 * (1.0 - eta2 * eta3);
        add(w0, w3, w0 + w1, w2, weight * jac, false, w0, w3, w0 + w1, w2);
    }
}
