// dropin_test.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A reference-style driver: it builds the reference's own Mesh2D, QuadratureRule
// and operators, and the dg::b200 drop-ins from include/wdg_b200.hpp with the
// same constructor arguments, then checks that the drop-ins give the reference's
// answers -- operator by operator, through the reference's own ode::RungeKutta4
// driving the GPU operators with host arrays (the examples/wave2d.cpp pattern),
// through the fused GPU stepper, and through WaveHoltz.  Exit status 0 = all
// within tolerance.  Built by `make -C oracle ref` into oracle/_ref/.
#include <cmath>
#include <cstdio>
#include <random>
#include <type_traits>
#include <vector>

#include "wavedg.hpp"
#include "wdg_b200.hpp"

using namespace dg;

static double rel(const std::vector<double> &a, const std::vector<double> &b)
{
    double num = 0, den = 0;
    for (size_t i = 0; i < a.size(); ++i)
    {
        num += (a[i] - b[i]) * (a[i] - b[i]);
        den += b[i] * b[i];
    }
    return std::sqrt(num / (den > 0 ? den : 1.0));
}

static int failures = 0;
static void report(const char *what, double err, double tol)
{
    const bool ok = err <= tol;
    std::printf("%-44s %.3e  (tol %.0e)  %s\n", what, err, tol, ok ? "ok" : "FAIL");
    failures += ok ? 0 : 1;
}

static Mesh2D perturbed_mesh(int n, unsigned seed)
{
    const int nv = (n + 1) * (n + 1);
    std::vector<double> xy(2 * nv);
    std::vector<int> q(4 * n * n);
    std::mt19937 gen(seed);
    std::uniform_real_distribution<double> U(-0.2, 0.2);
    const double h = 2.0 / n;
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i)
        {
            const bool inner = i > 0 && i < n && j > 0 && j < n;
            xy[2 * (i + (n + 1) * j)] = -1.0 + h * i + (inner ? U(gen) * h : 0.0);
            xy[2 * (i + (n + 1) * j) + 1] = -1.0 + h * j + (inner ? U(gen) * h : 0.0);
        }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
        {
            int *e = &q[4 * (i + n * j)];
            e[0] = i + (n + 1) * j;
            e[1] = i + 1 + (n + 1) * j;
            e[2] = i + 1 + (n + 1) * (j + 1);
            e[3] = i + (n + 1) * (j + 1);
        }
    return Mesh2D::from_vertices(nv, xy.data(), n * n, q.data());
}

int main()
{
    auto basis = QuadratureRule::quadrature_rule(5, QuadratureRule::GaussLobatto);
    Mesh2D mesh = perturbed_mesh(12, 7);
    const int ndof = 3 * 25 * mesh.n_elem();
    std::vector<int> bc(mesh.n_edges(FaceType::BOUNDARY), 1); // reflecting: the reference's WaveBC verbatim

    WaveEquation a(mesh, basis, true);
    WaveBC b(mesh, bc.data(), basis, true);
    MassMatrix<true> m(mesh, basis);
    b200::WaveEquation ga(mesh, basis, true);
    b200::WaveBC gb(mesh, bc.data(), basis, true);
    b200::MassMatrix gm(mesh, basis);

    std::mt19937 gen(11);
    std::normal_distribution<double> N01;
    std::vector<double> u(ndof);
    for (double &x : u)
        x = N01(gen);

    std::vector<double> r1(ndof, 0.0), r2(ndof, 0.0);
    a.action(u.data(), r1.data());
    ga.action(u.data(), r2.data());
    report("WaveEquation::action", rel(r2, r1), 1e-12);
    b.action(u.data(), r1.data());
    gb.action(u.data(), r2.data());
    report("WaveEquation + WaveBC::action", rel(r2, r1), 1e-12);
    m.inv(3, r1.data());
    gm.inv(3, r2.data());
    report("MassMatrix<true>::inv", rel(r2, r1), 1e-12);

    // the reference's RK4 driving (a) the reference operators, (b) the drop-ins on host arrays
    const double dt = 0.1 * mesh.min_h() / 25.0;
    ode::RungeKutta4 rk(ndof);
    auto f_ref = [&](double *dudt, const double, const double *v)
    {
        for (int i = 0; i < ndof; ++i)
            dudt[i] = 0.0;
        a.action(v, dudt);
        b.action(v, dudt);
        m.inv(3, dudt);
    };
    auto f_gpu = [&](double *dudt, const double, const double *v)
    {
        for (int i = 0; i < ndof; ++i)
            dudt[i] = 0.0;
        ga.action(v, dudt);
        gb.action(v, dudt);
        gm.inv(3, dudt);
    };
    std::vector<double> ur = u, ug = u, uf = u;
    double tr = 0.0, tg = 0.0, tf = 0.0;
    for (int s = 0; s < 10; ++s)
    {
        rk.step(dt, f_ref, tr, ur.data());
        rk.step(dt, f_gpu, tg, ug.data());
    }
    report("ode::RungeKutta4 over the drop-ins, 10 steps", rel(ug, ur), 1e-11);
    b200::WaveSystem sys(mesh, basis, bc.data());
    sys.rk4_steps(dt, tf, uf.data(), 10);
    report("fused GPU RK4, 10 steps", rel(uf, ur), 1e-11);
    report("time after 10 steps", std::abs(tf - tr), 1e-15);

    // WaveHoltz with reflecting walls (the reference class itself)
    Mesh2D small = perturbed_mesh(5, 3);
    std::vector<int> bc2(small.n_edges(FaceType::BOUNDARY), 1);
    const int nd2 = 3 * 25 * small.n_elem();
    LinearFunctional2D L(small, basis);
    std::vector<double> F(nd2);
    L.action(3, [](const double *x, double *o) { o[0] = 4.0 * std::exp(-((x[0] - 0.1) * (x[0] - 0.1) + (x[1] - 0.2) * (x[1] - 0.2)) / 0.08); o[1] = o[2] = 0.0; }, F.data());
    WaveHoltz wh(2.0, small, basis, bc2.data(), true);
    b200::WaveHoltz gwh(2.0, small, basis, bc2.data(), true);
    std::vector<double> p1(nd2), p2(nd2);
    wh.pi0(p1.data(), F.data());
    gwh.pi0(p2.data(), F.data());
    report("WaveHoltz::pi0", rel(p2, p1), 1e-12);
    std::vector<double> s1 = p1, s2 = p1;
    wh.S(s1.data());
    gwh.S(s2.data());
    report("WaveHoltz::S", rel(s2, s1), 1e-12);
    std::vector<double> H1(2 * nd2 / 3), H2(2 * nd2 / 3);
    wh.postprocess(H1.data(), s1.data());
    gwh.postprocess(H2.data(), s1.data());
    report("WaveHoltz::postprocess", rel(H2, H1), 1e-12);

    // approx_quad = false: the reference's exact-quadrature operators against the drop-ins
    {
        WaveEquation aq(mesh, basis, false);
        WaveBC bq(mesh, bc.data(), basis, false);
        MassMatrix<false> mq(mesh, basis);
        b200::WaveEquation gaq(mesh, basis, false);
        b200::WaveBC gbq(mesh, bc.data(), basis, false);
        b200::MassMatrix<false> gmq(mesh, basis);
        std::vector<double> q1(ndof, 0.0), q2(ndof, 0.0);
        aq.action(u.data(), q1.data());
        gaq.action(u.data(), q2.data());
        report("WaveEquation::action, approx_quad = false", rel(q2, q1), 1e-12);
        bq.action(u.data(), q1.data());
        gbq.action(u.data(), q2.data());
        report("+ WaveBC::action, approx_quad = false", rel(q2, q1), 1e-12);
        mq.inv(3, q1.data());
        gmq.inv(3, q2.data());
        report("MassMatrix<false>::inv", rel(q2, q1), 1e-12);
        std::vector<double> y1(ndof), y2(ndof);
        mq.action(3, u.data(), y1.data());
        gmq.action(3, u.data(), y2.data());
        report("MassMatrix<false>::action", rel(y2, y1), 1e-12);
        auto fq_ref = [&](double *dudt, const double, const double *v)
        {
            for (int i = 0; i < ndof; ++i)
                dudt[i] = 0.0;
            aq.action(v, dudt);
            bq.action(v, dudt);
            mq.inv(3, dudt);
        };
        auto fq_gpu = [&](double *dudt, const double, const double *v)
        {
            for (int i = 0; i < ndof; ++i)
                dudt[i] = 0.0;
            gaq.action(v, dudt);
            gbq.action(v, dudt);
            gmq.inv(3, dudt);
        };
        std::vector<double> vr = u, vg = u;
        double t1 = 0.0, t2 = 0.0;
        for (int s = 0; s < 5; ++s)
        {
            rk.step(dt, fq_ref, t1, vr.data());
            rk.step(dt, fq_gpu, t2, vg.data());
        }
        report("ode::RungeKutta4, exact quadrature, 5 steps", rel(vg, vr), 1e-11);
    }

    // WaveHoltz with approx_quad = false, reflecting walls: the reference's class against the drop-in
    {
        WaveHoltz whq(2.0, small, basis, bc2.data(), false);
        b200::WaveHoltz gwhq(2.0, small, basis, bc2.data(), false);
        std::vector<double> p1(nd2), p2(nd2);
        whq.pi0(p1.data(), F.data());
        gwhq.pi0(p2.data(), F.data());
        report("WaveHoltz::pi0, approx_quad = false", rel(p2, p1), 1e-12);
        std::vector<double> s1 = p1, s2 = p1;
        whq.S(s1.data());
        gwhq.S(s2.data());
        report("WaveHoltz::S, approx_quad = false", rel(s2, s1), 1e-12);
    }

    // the batched solver on the same two problems as two single solves (exact same periods)
    {
        b200::WaveSystem sa(small, basis, bc2.data()), sb(small, basis, bc2.data());
        b200::WaveHoltz wa(2.0, small, basis, bc2.data(), true), wb(3.0, small, basis, bc2.data(), true);
        std::vector<double> Wa(nd2, 0.0), Wb(nd2, 0.0), Ba(nd2, 0.0), Bb(nd2, 0.0), ra(1), rb(1);
        const int ia = wa.solve(F.data(), 1e-8, 40, Wa.data(), ra.data());
        const int ib = wb.solve(F.data(), 1e-8, 40, Wb.data(), rb.data());
        b200::WaveHoltzBatch batch({&sa, &sb}, {2.0, 3.0});
        const auto res = batch.solve({F.data(), F.data()}, {Ba.data(), Bb.data()}, 1e-8, 40);
        report("WaveHoltzBatch vs WaveHoltz::solve, omega 2", rel(Ba, Wa), 1e-10);
        report("WaveHoltzBatch vs WaveHoltz::solve, omega 3", rel(Bb, Wb), 1e-10);
        report("WaveHoltzBatch iteration counts", std::abs(res.iterations[0] - ia) + std::abs(res.iterations[1] - ib), 0.5);
    }

    // the nonlinear example's pattern (examples/cl2d.cpp, both settings of approx_quad): the
    // reference's DivF2D / EdgeFluxF2D / prolongators / MassMatrix with that example's Euler
    // flux and local Lax-Friedrichs flux, driven by ode::SSPRK3, against b200::EulerSystem
    auto euler_case = [&](auto approx)
    {
        constexpr bool AQ = decltype(approx)::value;
        const char *tag = AQ ? "approx_quad = true" : "approx_quad = false";
        const int nde = 4 * 25 * mesh.n_elem(), nI = mesh.n_edges(FaceType::INTERIOR),
                  nB = mesh.n_edges(FaceType::BOUNDARY);
        auto F = [](const double *, const double *q, double *fg)
        {
            const double rho = q[0], uu = q[1] / q[0], vv = q[2] / q[0], E = q[3];
            const double p = 0.4 * (E - 0.5 * rho * (uu * uu + vv * vv));
            fg[0] = rho * uu;
            fg[1] = rho * uu * uu + p;
            fg[2] = rho * uu * vv;
            fg[3] = uu * (E + p);
            fg[4] = rho * vv;
            fg[5] = rho * uu * vv;
            fg[6] = rho * vv * vv + p;
            fg[7] = vv * (E + p);
        };
        auto speed = [](const double *q)
        {
            const double rho = q[0], uu = q[1] / q[0], vv = q[2] / q[0], E = q[3];
            const double p = 0.4 * (E - 0.5 * rho * (uu * uu + vv * vv));
            return std::hypot(uu, vv) + std::sqrt(1.4 * p / rho);
        };
        auto llf = [&](const double *x, const double *nrm, const double *qL, const double *qR, double *fh)
        {
            double fL[8], fR[8];
            F(x, qL, fL);
            F(x, qR, fR);
            const double c = std::max(speed(qL), speed(qR));
            for (int d = 0; d < 4; ++d)
                fh[d] = 0.5 * nrm[0] * (fL[d] + fR[d]) + 0.5 * nrm[1] * (fL[4 + d] + fR[4 + d]) + 0.5 * c * (qL[d] - qR[d]);
        };
        DivF2D<AQ> div(mesh, basis);
        EdgeFluxF2D<AQ> fI(mesh, FaceType::INTERIOR, basis), fB(mesh, FaceType::BOUNDARY, basis);
        MassMatrix<AQ> me(mesh, basis);
        auto pI = make_face_prolongator(mesh, basis, FaceType::INTERIOR);
        auto pB = make_face_prolongator(mesh, basis, FaceType::BOUNDARY);
        std::vector<double> uI(5 * 4 * 2 * (size_t)nI), uB(5 * 4 * 2 * (size_t)nB);
        auto dudt = [&](double *out, double, const double *v)
        {
            for (int i = 0; i < nde; ++i)
                out[i] = 0.0;
            div.action(4, F, v, out);
            pI->action(4, v, uI.data());
            fI.action(4, llf, uI.data(), uI.data());
            for (double &x : uI)
                x = -x;
            pI->t(4, uI.data(), out);
            pB->action(4, v, uB.data());
            for (int e = 0; e < nB; ++e)
                for (int d = 0; d < 4; ++d)
                    for (int i = 0; i < 5; ++i)
                        uB[i + 5 * (d + 4 * (1 + 2 * (size_t)e))] = uB[i + 5 * (d + 4 * (0 + 2 * (size_t)e))];
            fB.action(4, llf, uB.data(), uB.data());
            for (double &x : uB)
                x = -x;
            pB->t(4, uB.data(), out);
            me.inv(4, out);
        };
        b200::EulerSystem<AQ> ge(mesh, basis);
        std::uniform_real_distribution<double> U01(0.0, 1.0);
        std::vector<double> q(nde);
        for (int k = 0; k < nde / 4; ++k)
        {
            const double rho = 1.0 + 0.2 * U01(gen), uu = 0.3 * N01(gen), vv = 0.3 * N01(gen), p = 1.0 + 0.2 * U01(gen);
            q[4 * k] = rho;
            q[4 * k + 1] = rho * uu;
            q[4 * k + 2] = rho * vv;
            q[4 * k + 3] = p / 0.4 + 0.5 * rho * (uu * uu + vv * vv);
        }
        std::vector<double> e1(nde), e2(nde);
        dudt(e1.data(), 0.0, q.data());
        ge.action(q.data(), e2.data());
        std::printf("Euler, %s:\n", tag);
        report("  time derivative (cl2d composition)", rel(e2, e1), 1e-12);
        const double dte = 0.1 * mesh.min_h() / 25.0;
        std::vector<double> qr = q, qg = q;
        double tr = 0.0, tg = 0.0;
        ode::SSPRK3 ssp(nde);
        for (int s = 0; s < 5; ++s)
            ssp.step(dte, dudt, tr, qr.data());
        ge.steps(dte, tg, qg.data(), 5);
        report("  ode::SSPRK3 vs b200::EulerSystem, 5 steps", rel(qg, qr), 1e-11);
    };
    euler_case(std::true_type{});
    euler_case(std::false_type{});

    // examples/advec2d.cpp as shipped: a Gauss-Legendre basis, approx_quad = false, the rotating
    // coefficient c = r (y, -x) projected by LinearFunctional2D and MassMatrix<false>::inv, and
    // ode::SSPRK3 on M^{-1} (Advection + AdvectionHomogeneousBC), against b200::Advection,
    // b200::AdvectionHomogeneousBC and b200::AdvectionSystem
    {
        auto gl = QuadratureRule::quadrature_rule(5, QuadratureRule::GaussLegendre);
        Mesh2D amesh = perturbed_mesh(8, 11);
        const int nd = 25 * amesh.n_elem();
        MassMatrix<false> am(amesh, gl);
        LinearFunctional2D LF(amesh, gl);
        std::vector<double> c(2 * (size_t)nd);
        auto coefficient = [](const double x[2], double cc[2])
        {
            const double r = std::hypot(x[0], x[1]);
            cc[0] = r * x[1];
            cc[1] = -r * x[0];
        };
        LF.action(2, coefficient, c.data());
        am.inv(2, c.data());
        Advection<false> adv(1, amesh, gl, c.data(), false);
        AdvectionHomogeneousBC<false> abc(1, amesh, gl, c.data(), false);
        auto dudt = [&](double *out, double, const double *v)
        {
            for (int i = 0; i < nd; ++i)
                out[i] = 0.0;
            adv.action(v, out);
            abc.action(v, out);
            am.inv(1, out);
        };
        b200::Advection<false> gadv(1, amesh, gl, c.data(), false);
        b200::AdvectionHomogeneousBC<false> gbc(1, amesh, gl, c.data(), false);
        b200::AdvectionSystem<false> gsys(1, amesh, gl, c.data(), false);
        std::vector<double> u(nd), r1(nd), r2(nd);
        for (double &x : u)
            x = N01(gen);
        for (int i = 0; i < nd; ++i)
            r1[i] = r2[i] = N01(gen);
        adv.action(u.data(), r1.data());
        gadv.action(u.data(), r2.data());
        std::printf("advection, Gauss-Legendre basis, approx_quad = false:\n");
        report("  Advection::action", rel(r2, r1), 1e-12);
        for (int i = 0; i < nd; ++i)
            r1[i] = r2[i] = N01(gen);
        abc.action(u.data(), r1.data());
        gbc.action(u.data(), r2.data());
        report("  AdvectionHomogeneousBC::action", rel(r2, r1), 1e-12);
        dudt(r1.data(), 0.0, u.data());
        gsys.action(u.data(), r2.data());
        report("  time derivative (advec2d composition)", rel(r2, r1), 1e-12);
        const double dta = 1.0 / 25.0 / M_SQRT2 * amesh.min_h();
        std::vector<double> ur = u, ug = u;
        double tr = 0.0, tg = 0.0;
        ode::SSPRK3 ssp(nd);
        for (int s = 0; s < 5; ++s)
            ssp.step(dta, dudt, tr, ur.data());
        gsys.steps(dta, tg, ug.data(), 5);
        report("  ode::SSPRK3 vs b200::AdvectionSystem, 5 steps", rel(ug, ur), 1e-11);
    }

    std::printf("%s\n", failures ? "DROP-IN FAILED" : "drop-in ok");
    return failures ? 1 : 0;
}
