"""Producer boundary of the reference's framework, mirrored for the host side.

Same names and behaviour as src/julia-serial/Framework: a ProductRegistry hands
out typed put/get tokens and refuses a type produced twice or consumed but never
produced (ProductRegistry.jl:8-24); an Event holds products by token
(EandES.jl:7-32); an EventSetup holds one product per type (EandES.jl:43-61);
plugin factories register producers by name (PluginFactory.jl:6-16,
ESPluginFactory.jl:6-16). The event loop itself is not part of this package.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable


@dataclass(frozen=True)
class EDPutTokenT:
    type: type
    index: int


@dataclass(frozen=True)
class EDGetTokenT:
    type: type
    index: int


class ProductRegistry:
    def __init__(self):
        self._produced: dict[type, int] = {}
        self._consumed: set[type] = set()

    def produces(self, t: type) -> EDPutTokenT:
        if t in self._produced:
            raise ValueError(f"{t.__name__} is already produced by another module")
        self._produced[t] = len(self._produced)
        return EDPutTokenT(t, self._produced[t])

    def consumes(self, t: type) -> EDGetTokenT:
        if t not in self._produced:
            raise ValueError(f"{t.__name__} is consumed but not produced by an earlier module")
        self._consumed.add(t)
        return EDGetTokenT(t, self._produced[t])

    def __len__(self) -> int:
        return len(self._produced)


class Event:
    def __init__(self, stream_id: int, event_id: int, registry: ProductRegistry):
        self.stream_id = stream_id
        self.event_id = event_id
        self.products: list[Any] = [None] * max(len(registry), 1)

    def get(self, token: EDGetTokenT):
        p = self.products[token.index]
        if p is None:
            raise KeyError(f"product {token.type.__name__} not in the event")
        return p

    def emplace(self, token: EDPutTokenT, obj) -> None:
        if token.index >= len(self.products):
            self.products.extend([None] * (token.index + 1 - len(self.products)))
        self.products[token.index] = obj


class EventSetup:
    def __init__(self):
        self._products: dict[type, Any] = {}

    def put(self, obj) -> None:
        t = type(obj)
        if t in self._products:
            raise ValueError(f"{t.__name__} already in the EventSetup")
        self._products[t] = obj

    def get(self, t: type):
        if t not in self._products:
            raise KeyError(f"{t.__name__} not in the EventSetup")
        return self._products[t]

    def has(self, t: type) -> bool:
        return t in self._products


class EDProducer:
    """Base of the event producers: __init__(registry) declares tokens, produce(event, es)."""

    def produce(self, event: Event, es: EventSetup) -> None:  # pragma: no cover - interface
        raise NotImplementedError


class ESProducer:
    """Base of the conditions producers: __init__(data_dir), produce(es)."""

    def produce(self, es: EventSetup) -> None:  # pragma: no cover - interface
        raise NotImplementedError


_ED_PLUGINS: dict[str, Callable[[ProductRegistry], EDProducer]] = {}
_ES_PLUGINS: dict[str, Callable[[str], ESProducer]] = {}


def add_plugin_module(name: str, ctor: Callable[[ProductRegistry], EDProducer]) -> None:
    _ED_PLUGINS[name] = ctor


def create_plugin_module(name: str, registry: ProductRegistry) -> EDProducer:
    return _ED_PLUGINS[name](registry)


def add_plugin(name: str, ctor: Callable[[str], ESProducer]) -> None:
    _ES_PLUGINS[name] = ctor


def create_plugin(name: str, data_dir: str) -> ESProducer:
    return _ES_PLUGINS[name](data_dir)


def plugin_names() -> tuple[list[str], list[str]]:
    return sorted(_ED_PLUGINS), sorted(_ES_PLUGINS)
