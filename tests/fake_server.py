"""A stand-in for the ISAAC server on 127.0.0.1: it accepts one client at a time,
splits what the client sends into its ``{"uid": n, ...} `` messages, records them,
and can answer with JSON objects (steering, ``done`` acknowledgements, errors)."""

from __future__ import annotations

import json
import socket
import threading
import time


class FakeServer:
    def __init__(self, ack: bool = True):
        self.ack = ack  # answer every message with {"done": uid + 1}
        self.listener = socket.socket(socket.AF_INET, socket.SOCK_STREAM)
        self.listener.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
        self.listener.bind(("127.0.0.1", 0))
        self.listener.listen(4)
        self.port = self.listener.getsockname()[1]
        self.messages: list[dict] = []
        self.raw: list[bytes] = []
        self.connection_of: list[int] = []  # per message: the connection (1, 2, ...) it came on
        self.connections = 0
        self.conn: socket.socket | None = None
        self._cv = threading.Condition()
        self._stop = False
        self._thread = threading.Thread(target=self._serve, daemon=True)
        self._thread.start()

    def _serve(self):
        while not self._stop:
            try:
                conn, _ = self.listener.accept()
            except OSError:
                return
            with self._cv:
                self.conn = conn
                self.connections += 1
                number = self.connections
                self._cv.notify_all()
            dec = json.JSONDecoder()
            buf = ""
            while True:
                try:
                    chunk = conn.recv(1 << 20)
                except OSError:
                    break
                if not chunk:
                    break
                buf += chunk.decode()
                while True:
                    s = buf.lstrip()
                    if not s:
                        buf = ""
                        break
                    try:
                        obj, end = dec.raw_decode(s)
                    except json.JSONDecodeError:
                        buf = s
                        break
                    with self._cv:
                        self.raw.append(s[:end].encode())
                        self.messages.append(obj)
                        self.connection_of.append(number)
                        self._cv.notify_all()
                    buf = s[end:]
                    if self.ack and isinstance(obj, dict) and "uid" in obj:
                        self.send({"done": obj["uid"] + 1})
            with self._cv:
                if self.conn is conn:
                    self.conn = None
            conn.close()

    def send(self, obj) -> None:
        """Send one JSON value (or raw text) to the connected client."""
        data = obj.encode() if isinstance(obj, str) else json.dumps(obj).encode()
        with self._cv:
            conn = self.conn
        if conn is not None:
            conn.sendall(data)

    def wait_messages(self, n: int, timeout: float = 10.0) -> list[dict]:
        end = time.time() + timeout
        with self._cv:
            while len(self.messages) < n:
                left = end - time.time()
                if left <= 0:
                    raise TimeoutError(f"{len(self.messages)} of {n} messages")
                self._cv.wait(left)
            return list(self.messages)

    def wait_connections(self, n: int, timeout: float = 10.0) -> None:
        end = time.time() + timeout
        with self._cv:
            while self.connections < n:
                left = end - time.time()
                if left <= 0:
                    raise TimeoutError("no connection")
                self._cv.wait(left)

    def drop(self) -> None:
        """Close the current connection from the server side."""
        with self._cv:
            conn, self.conn = self.conn, None
        if conn is not None:
            try:
                conn.shutdown(socket.SHUT_RDWR)
            except OSError:
                pass
            conn.close()

    def close(self) -> None:
        self._stop = True
        self.drop()
        self.listener.close()
