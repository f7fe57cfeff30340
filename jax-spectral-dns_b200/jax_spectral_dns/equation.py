"""Equation base class with the reference's field registry and time loop
(jax_spectral_dns/equation.py in dakling/jax-spectral-dns)."""
from __future__ import annotations

import os
import time
from typing import Any, Callable, Dict, List, Optional

from .field import Field


def print_verb(*args, verbosity_level: int = 1, debug: bool = False, **kwargs) -> None:
    """Print when Equation.verbosity_level >= verbosity_level (equation.py:56-75)."""
    if Equation.verbosity_level >= verbosity_level:
        print(*args, **kwargs)


class Equation:
    name = "equation"
    write_intermediate_output = False
    write_entire_output = False
    verbosity_level: int = int(os.environ.get("JAX_SPECTRAL_DNS_VERBOSITY_LEVEL", 1))

    def __init__(self, domain, *fields, **params: Any):
        self._dt = float(params.get("dt", 1e-2))
        self._domain = domain
        self.fields: Dict[str, List[Any]] = {}
        self.time_step: int = 0
        self.time: float = 0.0
        self.before_time_step_fn: Optional[Callable] = None
        self.after_time_step_fn: Optional[Callable] = None
        self.post_process_fn: Optional[Callable] = None
        self.end_time = params.get("end_time", 0.0)
        self.max_iter = params.get("max_iter", 1000)
        for f in fields:
            nm = f.get_name()
            self.fields[nm] = [f]

    @classmethod
    def initialize(cls, cleanup: bool = True) -> None:
        Field.initialize(cleanup)

    @classmethod
    def find_suitable_dt(cls, domain, max_cfl: float = 0.7, U_max=(1.0, 1e-10, 1e-10),
                         end_time: Optional[float] = None, safety_factor: float = 0.9) -> float:
        """Time step for a CFL number (equation.py:114-162): the smallest
        max_cfl * (extent / cells) / U_max over the directions, times the safety
        factor; with an end time, the step count is raised until its median
        factor splits it into inner and outer steps no worse than the square
        root, and dt = end_time / steps."""
        dT = [abs(max_cfl * (domain.get_extent(i) / domain.number_of_cells(i)) / U_max[i])
              for i in domain.all_dimensions()]
        dt = safety_factor * min(dT)
        if end_time is None:
            return dt

        def median_factor(n: int) -> int:
            factors = sorted(f for i in range(1, int(n ** 0.5) + 1) if n % i == 0 for f in (i, n // i))
            return factors[len(factors) // 2]

        steps = max(0, int(end_time / dt))

        def bad(n: int) -> bool:
            outer = n // median_factor(n)
            return abs(n ** 0.5) - outer > outer

        while bad(steps):
            steps += 1
        return end_time / steps

    def get_dt(self) -> float:
        return self._dt

    def get_domain(self):
        return self._domain

    def get_field(self, name: str, index: int):
        try:
            return self.fields[name][index]
        except KeyError:
            raise KeyError("Expected field named " + name + " in " + self.name + ".")

    def get_fields(self, name: str):
        try:
            return self.fields[name]
        except KeyError:
            raise KeyError("Expected field named " + name + " in " + self.name + ".")

    def get_initial_field(self, name: str):
        return self.get_field(name, 0)

    def get_latest_field(self, name: str):
        return self.get_field(name, -1)

    def get_number_of_fields(self, name: str) -> int:
        return len(self.get_fields(name))

    def set_field(self, name: str, index: int, field) -> None:
        self.fields[name][index] = field

    def set_initial_field(self, name: str, field) -> None:
        self.clear_field(name)
        self.append_field(name, field)

    def append_field(self, name: str, field, in_place: bool = True) -> None:
        if name not in self.fields:
            raise KeyError("Expected field named " + name + " in " + self.name + ".")
        if in_place and len(self.fields[name]) > 0:
            self.fields[name][-1] = field
        else:
            self.fields[name].append(field)
        self.fields[name][-1].name = name

    def add_field(self, name: str, field=None) -> None:
        assert name not in self.fields, "Field " + name + " already exists!"
        self.fields[name] = [] if field is None else [field]

    def clear_field(self, name: str) -> None:
        self.fields[name] = []

    def activate_jit(self) -> None:
        Field.activate_jit_ = True

    def deactivate_jit(self) -> None:
        Field.activate_jit_ = False

    def all_dimensions(self):
        return range(3)

    def done(self) -> bool:
        iteration_done = self.max_iter is not None and self.time_step > self.max_iter
        time_done = self.end_time is not None and self.time >= self.end_time + self.get_dt() + 1e-40
        return iteration_done or time_done

    def set_before_time_step_fn(self, fn) -> None:
        self.before_time_step_fn = fn

    def set_after_time_step_fn(self, fn) -> None:
        self.after_time_step_fn = fn

    def set_post_process_fn(self, fn) -> None:
        self.post_process_fn = fn

    def before_time_step(self) -> None:
        if self.before_time_step_fn is not None:
            self.before_time_step_fn(self)

    def after_time_step(self) -> None:
        if self.after_time_step_fn is not None:
            self.after_time_step_fn(self)

    def update_time(self) -> None:
        self.time += self.get_dt()
        self.time_step += 1

    def prepare(self) -> None:
        pass

    def perform_time_step(self, *args, **kwargs):
        raise NotImplementedError()

    def solve_scan(self):
        raise NotImplementedError()

    def solve(self):
        """With jit active: the whole horizon in one device loop (solve_scan);
        otherwise a host loop of single steps with the before/after hooks
        (equation.py:334-427)."""
        self.prepare()
        if Field.activate_jit_:
            t0 = time.time()
            out = self.solve_scan()
            print_verb("Took " + "{:.3e}".format(time.time() - t0) + " seconds", verbosity_level=2)
            return out
        while not self.done():
            self.before_time_step()
            self.perform_time_step(None, None, self.time_step)
            self.update_time()
            self.after_time_step()
        return None
