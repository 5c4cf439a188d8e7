/* hpGEM-side adapter: an HpgemAPISimplified<DIM> whose time step runs on the GPU.
 *
 * Header-only, compiled inside an hpGEM application (it includes hpGEM's kernel
 * headers and links libhpgem_b200.so).  An application derives from
 * hpgem_b200::GpuSimplified<DIM> instead of hpgem::Base::HpgemAPISimplified<DIM>,
 * sets physics_ / advection_ / cInv_ in its constructor and calls solve()
 * unchanged:
 *   - computeOneTimeStep(time, dt) (HpgemAPISimplified_Impl.h:788-820) becomes
 *     hgg_step: the stage loop, both face sides, the mass solve and the RK update
 *     run on the device; the first call builds the device problem from hpGEM's own
 *     mesh, basis, quadrature rules and Butcher tableau (hgg_create) and uploads
 *     the initial solution hpGEM projected (hgg_set_state);
 *   - tasksAfterSolving() first copies the solution back into every element's
 *     time-integration vector (hgg_get_state), so hpGEM's error norms and output
 *     writers read the GPU result.
 * A failed call ends in logger(ERROR, ...), hpGEM's own convention.
 *
 * The descriptor takes the reference tabulations hpGEM itself integrates with:
 * the element rule of the first element (all elements share shape and order),
 * the basis and its reference gradients at those points, per element the
 * Jacobian of its (affine) reference-to-physical map, per face the left/right
 * elements and local faces, the face rule, the basis of each side at the face
 * points mapped into that side's reference element (mapRefFaceToRefElemL / R,
 * FaceGeometry.h:362-395; one tabulation per distinct (side, local face,
 * face-to-face map) triple) and the face normal of length area ratio
 * (getNormalVector, FaceGeometry.h:412-459).  Faces must be internal (periodic
 * meshes): the matrix-free path has no boundary faces. */
#pragma once

#include <cstdint>
#include <map>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "Base/Element.h"
#include "Base/Face.h"
#include "Base/HpgemAPISimplified.h"
#include "Base/MeshManipulator.h"
#include "Geometry/PointReference.h"
#include "Geometry/ReferenceGeometry.h"
#include "Integration/QuadratureRules/GaussQuadratureRule.h"
#include "Logger.h"
#include "hpgem_b200.h"

namespace hpgem_b200 {

template <std::size_t DIM>
class GpuSimplified : public hpgem::Base::HpgemAPISimplified<DIM> {
   public:
    using Base = hpgem::Base::HpgemAPISimplified<DIM>;
    using Base::Base;

    ~GpuSimplified() override {
        if (h_) hgg_destroy(h_);
    }

    // hpGEM's solve() calls this once per time step; it now runs on the GPU.
    void computeOneTimeStep(double &time, const double dt) override {
        upload_once();
        check(hgg_step(h_, &time, dt, 1));
        dirty_ = true;  // the element vectors are stale until the next download
    }

    void tasksAfterSolving() override {
        download();
        Base::tasksAfterSolving();
    }

   protected:
    int physics_ = HGG_PHYSICS_ADVECTION;  // or HGG_PHYSICS_WAVE / HGG_PHYSICS_WAVE_UPWIND
    double advection_[3] = {0.0, 0.0, 0.0};
    double cInv_ = 1.0;
    int precision_ = HGG_PRECISION_FP64;

    void check(int rc) const {
        if (rc != 0) hpgem::logger(hpgem::ERROR, "hpgem_b200: %", hgg_last_error(h_));
    }

    static int shape_of(hpgem::Geometry::ReferenceGeometryType t) {
        using T = hpgem::Geometry::ReferenceGeometryType;
        switch (t) {
            case T::LINE: return HGG_SHAPE_LINE;
            case T::TRIANGLE: return HGG_SHAPE_TRIANGLE;
            case T::SQUARE: return HGG_SHAPE_SQUARE;
            case T::TETRAHEDRON: return HGG_SHAPE_TETRAHEDRON;
            case T::CUBE: return HGG_SHAPE_CUBE;
            default: return -1;
        }
    }

    // The device problem from hpGEM's own objects, and the initial solution.
    void upload_once() {
        if (h_) return;
        auto *mesh = this->meshes_[0];
        std::vector<hpgem::Base::Element *> elements;
        std::unordered_map<const hpgem::Base::Element *, int64_t> index;
        for (hpgem::Base::Element *el : mesh->getElementsList()) {
            index[el] = (int64_t)elements.size();
            elements.push_back(el);
        }
        const hpgem::Base::Element *e0 = elements.front();
        const std::size_t nB = e0->getNumberOfBasisFunctions();

        // element rule (order 2p + 1, Element.cpp:89-98): weights, basis, reference gradients
        const hpgem::QuadratureRules::GaussQuadratureRule *rule = e0->getGaussQuadratureRule();
        std::vector<double> w, phi, dphi;
        for (std::size_t q = 0; q < rule->getNumberOfPoints(); ++q) {
            w.push_back(rule->weight(q));
            const hpgem::Geometry::PointReference<DIM> &p = rule->getPoint(q);
            for (std::size_t j = 0; j < nB; ++j) {
                phi.push_back(e0->basisFunction(j, p));
                const auto g = e0->basisFunctionDeriv(j, p);
                for (std::size_t d = 0; d < DIM; ++d) dphi.push_back(g[d]);
            }
        }
        // per element: the Jacobian of the affine map, J[r][c] = dx_r / dxi_c
        std::vector<double> jac;
        for (const hpgem::Base::Element *el : elements) {
            const hpgem::Geometry::PointReference<DIM> &c = el->getReferenceGeometry()->getCenter();
            const auto J = el->calcJacobian(c);
            for (std::size_t r = 0; r < DIM; ++r)
                for (std::size_t k = 0; k < DIM; ++k) jac.push_back(J(r, k));
        }
        // faces: elements, local faces, tabulation per (side, local face, face-to-face map), normals
        std::vector<int64_t> faceEl;
        std::vector<int32_t> faceLocal, faceTab;
        std::vector<double> faceW, faceTabs, normals;
        std::map<std::tuple<int, std::size_t, std::size_t>, int32_t> tabs;
        const hpgem::QuadratureRules::GaussQuadratureRule *frule = nullptr;
        for (const hpgem::Base::Face *f : mesh->getFacesList()) {
            if (!f->isInternal()) hpgem::logger(hpgem::ERROR, "hpgem_b200: the GPU path takes periodic meshes only");
            if (!frule) {
                frule = f->getGaussQuadratureRule();
                for (std::size_t q = 0; q < frule->getNumberOfPoints(); ++q) faceW.push_back(frule->weight(q));
            }
            const hpgem::Base::Element *sides[2] = {f->getPtrElementLeft(), f->getPtrElementRight()};
            const std::size_t local[2] = {f->localFaceNumberLeft(), f->localFaceNumberRight()};
            for (int s = 0; s < 2; ++s) {
                faceEl.push_back(index.at(sides[s]));
                faceLocal.push_back((int32_t)local[s]);
                const auto key = std::make_tuple(s, local[s], s == 0 ? std::size_t(0) : f->getFaceToFaceMapIndex());
                auto it = tabs.find(key);
                if (it == tabs.end()) {
                    it = tabs.emplace(key, (int32_t)tabs.size()).first;
                    for (std::size_t q = 0; q < frule->getNumberOfPoints(); ++q) {
                        const hpgem::Geometry::PointReference<DIM - 1> &pf = frule->getPoint(q);
                        const hpgem::Geometry::PointReference<DIM> pe =
                            s == 0 ? f->mapRefFaceToRefElemL(pf) : f->mapRefFaceToRefElemR(pf);
                        for (std::size_t j = 0; j < nB; ++j) faceTabs.push_back(sides[s]->basisFunction(j, pe));
                    }
                }
                faceTab.push_back(it->second);
            }
            const hpgem::Geometry::PointReference<DIM - 1> &p0 = frule->getPoint(0);
            const auto n = f->getNormalVector(p0);  // affine: constant on the face
            for (std::size_t d = 0; d < DIM; ++d) normals.push_back(n[d]);
        }

        hgg_problem_desc d{};
        d.dim = (int32_t)DIM;
        d.shape = shape_of(e0->getReferenceGeometry()->getGeometryType());
        d.order = (int32_t)this->polynomialOrder_;
        d.n_vars = (int32_t)this->configData_->numberOfUnknowns_;
        d.physics = physics_;
        d.precision = precision_;
        for (int i = 0; i < 3; ++i) d.advection[i] = advection_[i];
        d.c_inv = cInv_;
        d.n_elements = (int64_t)elements.size();
        d.n_basis = (int32_t)nB;
        d.n_quad = (int32_t)w.size();
        d.quad_weights = w.data();
        d.basis_values = phi.data();
        d.basis_grads = dphi.data();
        d.n_face_quad = (int32_t)faceW.size();
        d.face_weights = faceW.data();
        d.n_face_tabs = (int32_t)tabs.size();
        d.face_tabs = faceTabs.data();
        d.jacobians = jac.data();
        d.n_faces = (int64_t)(faceEl.size() / 2);
        d.face_elements = faceEl.data();
        d.face_local = faceLocal.data();
        d.face_tab_index = faceTab.data();
        d.face_normals = normals.data();
        const hpgem::TimeIntegration::ButcherTableau *bt = this->ptrButcherTableau_;
        const std::size_t S = bt->getNumberOfStages();
        std::vector<double> a(S * S, 0.0), b, c;
        for (std::size_t i = 0; i < S; ++i) {
            for (std::size_t j = 0; j < i; ++j) a[i * S + j] = bt->getA(i, j);
            b.push_back(bt->getB(i));
            c.push_back(bt->getC(i));
        }
        d.n_stages = (int32_t)S;
        d.rk_a = a.data();
        d.rk_b = b.data();
        d.rk_c = c.data();
        check(hgg_create(&d, &h_));

        // the initial solution hpGEM projected (setInitialSolution) -> device
        std::vector<double> u;
        for (const hpgem::Base::Element *el : elements) {
            const auto &v = el->getTimeIntegrationVector(this->solutionVectorId_);
            u.insert(u.end(), v.data(), v.data() + v.size());
        }
        check(hgg_set_state(h_, 0, u.data()));
    }

    // device -> every element's time-integration vector
    void download() {
        if (!dirty_ || !h_) return;
        std::vector<double> u((std::size_t)hgg_vector_length(h_));
        check(hgg_get_state(h_, 0, u.data()));
        std::size_t off = 0;
        for (hpgem::Base::Element *el : this->meshes_[0]->getElementsList()) {
            auto &v = el->getTimeIntegrationVector(this->solutionVectorId_);
            for (std::size_t i = 0; i < v.size(); ++i) v[i] = u[off + i];
            off += v.size();
        }
        dirty_ = false;
    }

   private:
    hgg_handle *h_ = nullptr;
    bool dirty_ = false;
};

}  // namespace hpgem_b200
