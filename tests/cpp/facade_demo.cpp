// Reference-style client code against the host facade (ne/world.hpp): the
// README example and the stacking selftest scenario, stepped on the device.
// Prints one line per check; exit status 0 iff all pass.
#include <cmath>
#include <cstdio>

#include "ne/world.hpp"

static int g_fail = 0;
static void check(bool ok, const char* what) {
    std::printf("[%s] %s\n", ok ? "PASS" : "FAIL", what);
    if (!ok) ++g_fail;
}

int main() {
    {   // README.md:61-72
        ne::PhysicsWorld w;
        w.setGravity({0.0, -9.81, 0.0});
        w.setTimestep(1.0 / 60.0);
        w.setOpenBoundary(true);
        w.setRestitution(0.2);
        w.setFriction(0.5);
        w.makeStatic(w.addBox({0.0, -1.0, 0.0}, {}, {50.0, 1.0, 50.0}, 1.0));
        ne::BodyId ball = w.addSphere({0.0, 10.0, 0.0}, 0.5, 1.0);
        for (int i = 0; i < 600; ++i) w.step();
        const double y = w.position(ball).y;
        std::printf("readme y = %.17g\n", y);
        check(y == 0.4890999999999725, "README example: ball rests at the reference's exact y");
    }
    {   // two-box stack (the reference selftest's stacking scenario)
        ne::PhysicsWorld pw;
        pw.setBox(1e6, false);
        pw.setTimestep(1.0 / 240.0);
        pw.setGravity(ne::V3{0, -10, 0});
        pw.setRestitution(0.0);
        pw.setFriction(0.6);
        pw.makeStatic(pw.addBox(ne::V3{0, -1, 0}, ne::Q{1, 0, 0, 0}, ne::V3{20, 1, 20}, 1.0));
        ne::BodyId lo = pw.addBox(ne::V3{0, 1.05, 0}, ne::Q{1, 0, 0, 0}, ne::V3{1, 1, 1}, 1.0);
        ne::BodyId hi = pw.addBox(ne::V3{0, 3.10, 0}, ne::Q{1, 0, 0, 0}, ne::V3{1, 1, 1}, 1.0);
        pw.world().stepDevice(4000);
        pw.world().syncFromDevice();
        const double yl = pw.position(lo).y, yh = pw.position(hi).y;
        check(yl > 0.85 && yl < 1.2, "stack: lower box rests on the floor");
        check(yh > 2.7 && yh < 3.3, "stack: upper box rests on the lower");
        check(pw.velocity(hi).norm() < 0.3, "stack: at rest");
    }
    {   // determinism + swap-and-pop removal
        auto run = [](bool removeOne) {
            ne::PhysicsWorld pw;
            pw.setBox(8.0, true);
            pw.setTimestep(5e-3);
            ne::BodyId ids[40];
            for (int i = 0; i < 40; ++i) {
                ids[i] = pw.addSphere(ne::V3{-6.0 + 0.3 * i, std::sin(1.7 * i) * 5.0, std::cos(2.3 * i) * 5.0}, 0.5, 1.0);
                pw.setVelocity(ids[i], ne::V3{std::cos(0.9 * i), std::sin(1.1 * i), 0.5});
            }
            if (removeOne) pw.remove(ids[7]);
            for (int s = 0; s < 200; ++s) pw.step();
            return pw.position(ids[39]);
        };
        const ne::V3 a = run(false), b = run(false);
        check(a.x == b.x && a.y == b.y && a.z == b.z, "determinism: identical runs are bit-identical");
        check(run(true).norm() > 0.0, "remove: swap-and-pop keeps handles valid");
    }
    {   // a sphere and a box on a two-triangle floor mesh (the reference's mesh self-test setting)
        ne::PhysicsWorld pw;
        pw.setBox(1000.0, false);
        pw.setTimestep(1.0 / 240.0);
        pw.setGravity(ne::V3{0, -10, 0});
        pw.setRestitution(0.0);
        pw.setFriction(0.5);
        pw.addMesh(ne::V3{0, 0, 0}, ne::Q{1, 0, 0, 0}, {{-10, 0, -10}, {10, 0, -10}, {10, 0, 10}, {-10, 0, 10}},
                   {0, 1, 2, 0, 2, 3});
        ne::BodyId ball = pw.addSphere(ne::V3{1, 5, 1}, 0.5, 1.0);
        ne::BodyId bx = pw.addBox(ne::V3{-3, 5, -2}, ne::Q{1, 0, 0, 0}, ne::V3{0.5, 0.5, 0.5}, 1.0);
        pw.world().stepDevice(1500);
        pw.world().syncFromDevice();
        check(std::fabs(pw.position(ball).y - 0.5) < 0.05, "mesh: sphere rests on the mesh floor");
        check(std::fabs(pw.position(bx).y - 0.5) < 0.08, "mesh: box rests on the mesh floor");
    }
    {   // a dumbbell compound on a floor box (the reference's compound self-test setting)
        ne::PhysicsWorld pw;
        pw.setBox(1000.0, false);
        pw.setTimestep(1.0 / 240.0);
        pw.setGravity(ne::V3{0, -10, 0});
        pw.setRestitution(0.0);
        pw.setFriction(0.5);
        pw.makeStatic(pw.addBox(ne::V3{0, -1, 0}, ne::Q{1, 0, 0, 0}, ne::V3{20, 1, 20}, 1.0));
        ne::BodyId db = pw.addCompound(ne::V3{0, 5, 0}, ne::Q{1, 0, 0, 0},
                                       {ne::ChildShape::sphere(ne::V3{-1, 0, 0}, 0.5),
                                        ne::ChildShape::sphere(ne::V3{1, 0, 0}, 0.5)}, 1.0);
        pw.world().stepDevice(1500);
        pw.world().syncFromDevice();
        check(std::fabs(pw.position(db).y - 0.5) < 0.05, "compound: dumbbell rests on both spheres");
        check(pw.velocity(db).norm() < 0.1, "compound: comes to rest");
    }
    std::printf("%d failed\n", g_fail);
    return g_fail == 0 ? 0 : 1;
}
