// The C ABI's opaque handles that hold host pipeline state.
#pragma once
#include "bake.h"

struct lb_bake {
    lb::Scene scene;
    lb::Bake bake;
};

struct lb_plan;
// The results of a plan's last launch as a bake (downloads, the cache writes): bake_device.cu.
lb::Bake lb_plan_collect(lb_plan &p);
const lb::Scene &lb_plan_scene(const lb_plan &p);
